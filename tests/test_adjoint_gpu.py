"""GPU reverse mode (blaze_ens_adj_*) against the FP64 reverse sweep of the
restatement, which tests/test_adjoint_oracle.py pins to central finite
differences.

Case: two box systems (40 and 60 spheres) thrown at random velocities,
200 steps of dt = 1e-5 s, checkpoints every 64 steps (the backward
recomputes four segments).  The GPU's forward equals the FP32 restatement's
bit for bit, and its reverse sweep equals the FP32 restatement's reverse
sweep within 1e-4 (the summation order of the reverse differs).

Against the FP64 reverse sweep the comparison runs over 120 steps, bound
1e-3: the gradients are pathwise (the derivative along the contact onsets
and stick/slip states the trajectory took), and somewhere between 120 and
160 steps of this case one such decision comes out differently in FP32 and
FP64 (a contact whose overlap crosses zero within the rounding); from there
the two precisions differentiate different branches and their gradients
part by O(1) (measured: 1.6e-4 of the largest component at 120 steps, 0.6
at 160; with the previous overlap arithmetic the flip came at 240).  That is
the active-branch nature of the derivative, not an arithmetic error.
"""
import numpy as np
import pytest

from bindings import EnsRestated
from blaze import device
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
    return _gpu_grads(case, T)


T_F64 = 120   # steps of the FP64 comparison (before the first branch flip of this case)


def _gpu_grads(case, steps):
    S, W, p, r, v0, wx, wv = case
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.02, max_nbr=32, use_graph=0)
    ens.set_state(p, r, v0)
    adj = E.Adjoint(ens, steps, SEG)
    assert adj.forward() == 0
    st = ens.state()
    gx, gv0, gw0, gc = adj.backward(wx[st["pid"]], wv[st["pid"]], None)
    adj.close()
    ens.close()
    return st, gx, gv0, gw0, gc


@pytest.fixture(scope="module", params=["f32", "f64"])
def oracle_grads(case, request):
    S, W, p, r, v0, wx, wv = case
    steps = T if request.param == "f32" else T_F64
    o = EnsRestated(S, W, 1, 1e-5, 0.02, 32, precision=request.param)
    o.set_state(p, r, v0)
    assert o.adj_record(steps) == 0
    st = o.state()
    dx0, dv0, dw0, th = o.adj_reverse(wx[st["pid"]], wv[st["pid"]], np.zeros(p.shape))
    return dx0, dv0, dw0, th, request.param


@pytest.fixture(scope="module")
def gpu_grads_f64_horizon(case):
    return _gpu_grads(case, T_F64)


def grads_for(oracle_grads, gpu_grads, gpu_grads_f64_horizon):
    return gpu_grads if oracle_grads[4] == "f32" else gpu_grads_f64_horizon


TOL = {"f32": 1e-4, "f64": 1e-3}
# the law-constant gradients are sums over every contact of every step with
# cancellation between them (measured against FP64 at 120 steps: up to
# 5e-3 relative, for kt of the 60-sphere system)
TOL_LAW = {"f32": 1e-4, "f64": 1e-2}


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
def test_initial_state_gradient(gpu_grads, gpu_grads_f64_horizon, oracle_grads, k, name):
    g = grads_for(oracle_grads, gpu_grads, gpu_grads_f64_horizon)[1 + k].astype(np.float64)
    o = oracle_grads[k]
    scale = np.abs(o).max()
    assert scale > 0
    err = np.abs(g - o).max() / scale
    prec = oracle_grads[4]
    print("%s gradient vs %s reverse sweep: max error %.2e of the largest component"
          % (name, prec, err))
    assert err < TOL[prec]


def test_law_constant_gradient(gpu_grads, gpu_grads_f64_horizon, oracle_grads):
    g = grads_for(oracle_grads, gpu_grads, gpu_grads_f64_horizon)[4]
    o = oracle_grads[3]
    rel = np.abs(g - o) / np.maximum(np.abs(o), 1e-30)
    prec = oracle_grads[4]
    print("law-constant gradients vs %s, relative error per (system, constant):\n" % prec, rel)
    assert np.all(rel < TOL_LAW[prec]), rel


def run_with_tape(case, **kw):
    S, W, p, r, v0, wx, wv = case
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.02, max_nbr=32, use_graph=0)
    ens.set_state(p, r, v0)
    adj = E.Adjoint(ens, T, SEG, **kw)
    assert adj.forward() == 0
    info = adj.tape_info()
    st = ens.state()
    out = adj.backward(wx[st["pid"]], wv[st["pid"]], None)
    info_after = adj.tape_info()
    adj.close()
    ens.close()
    return out, info, info_after


def assert_same_grads(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_tape_holding_every_segment(case, gpu_grads):
    """A budget that holds the whole run: the forward records all four
    segments, the backward recomputes none, and the gradients are those of
    the one-segment tape bit for bit (a recomputed segment reproduces the
    forward's tape exactly)."""
    out, info, _ = run_with_tape(case, tape_bytes=64 << 20)
    assert info[1] == 4, info
    assert_same_grads(out, gpu_grads[1:])


def state_bytes(n, steps):
    """Arena bytes of `steps` recorded steps' dense blocks (15 words per
    particle, rounded up to 4 words)."""
    return 4 * ((15 * n + 3) // 4 * 4) * steps


def test_tape_ring(case, gpu_grads):
    """An arena with room for one 64-step segment and its pools: the forward
    records the last two segments (their states fit), the last one wrapping
    to the start of the arena when the one before leaves no room; the
    backward reverses what is left, recomputes the rest, and the gradients
    are unchanged bit for bit."""
    n = len(case[2])
    _, _, full = run_with_tape(case, tape_bytes=64 << 20)
    pool_max = full[2]
    assert pool_max > 0
    out, info, _ = run_with_tape(case, arena_bytes=state_bytes(n, SEG) + pool_max + 1024)
    assert 1 <= info[1] < 4, info
    assert_same_grads(out, gpu_grads[1:])


def test_tape_pool_overflow(case):
    """Pool space for half the largest segment: the recording kernels find
    that their reservations do not fit and write nothing, and the backward
    reports it (-2) instead of reversing a segment it could not record."""
    n = len(case[2])
    _, _, full = run_with_tape(case, tape_bytes=64 << 20)
    S, W, p, r, v0, wx, wv = case
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.02, max_nbr=32, use_graph=0)
    ens.set_state(p, r, v0)
    adj = E.Adjoint(ens, T, SEG, arena_bytes=state_bytes(n, SEG) + full[2] // 2)
    assert adj.forward() == 0
    assert adj.tape_info()[1] < 4
    st = ens.state()
    with pytest.raises(device.BlazeError):
        adj.backward(wx[st["pid"]], wv[st["pid"]], None)
    adj.close()
    ens.close()


def test_tape_too_small_for_a_segment(case):
    S, W, p, r, v0, wx, wv = case
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.02, max_nbr=32, use_graph=0)
    with pytest.raises(device.BlazeError):
        E.Adjoint(ens, T, SEG, tape_bytes=1 << 10)
    ens.close()
