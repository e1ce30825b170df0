"""The reverse sweep of the ensemble restatement (FP64, oracle/ens_oracle.c)
against central finite differences of its forward.

The reverse sweep is the discrete adjoint of the step: the exact derivative
of the arithmetic on the branch each contact took (in contact or not, stick
or slip, history turned into the tangent plane or not), so the derivative at
a contact onset or a stick/slip switch is the one of the active branch.  A
finite difference that straddles such a switch would disagree; with h = 1e-6
relative none does here, and the agreement is ~1e-6 relative.

Case: two box systems (40 and 60 spheres) thrown at random velocities for
200 steps of dt = 1e-5 s -- pair and wall contacts, Coulomb slip, re-sorts
with history carried over.  Loss: a random linear functional of the final
positions and velocities.
"""
import numpy as np
import pytest

from bindings import EnsRestated
from blaze import calibrate, synth

T = 200


@pytest.fixture(scope="module")
def case():
    S, W, p, r = synth.box_ensemble([40, 60], seed=4, mus=[0.3, 0.6], restitutions=[0.5, 0.8],
                                    height_factor=4.0)
    rng = np.random.default_rng(0)
    v0 = rng.normal(scale=30.0, size=p.shape)
    wx = rng.normal(size=p.shape)
    wv = rng.normal(size=p.shape) * 1e-2
    return S, W, p.astype(np.float64), r.astype(np.float64), v0, wx, wv


def run(case, v=None, consts=None, steps=T, record=False):
    S, W, p, r, v0, wx, wv = case
    o = EnsRestated(S, W, 1, 1e-5, 0.02, 32, precision="f64")
    if consts is not None:
        for s, c in enumerate(consts):
            o.set_constants(s, c)
    o.set_state(p, r, v0 if v is None else v)
    if record:
        assert o.adj_record(steps) == 0
    else:
        assert o.step(steps) == 0
    return o


def loss(case, o):
    wx, wv = case[5], case[6]
    st = o.state()
    order = np.argsort(st["pid"])
    return float(np.sum(wx * st["pos"][order]) + np.sum(wv * st["vel"][order]))


@pytest.fixture(scope="module")
def adjoint(case):
    o = run(case, record=True)
    st = o.state()
    wx, wv = case[5], case[6]
    gx = wx[st["pid"]]
    gv = wv[st["pid"]]
    rebuilds = o.num_rebuilds()
    dx0, dv0, dw0, th = o.adj_reverse(gx, gv, np.zeros_like(gx))
    base = [o.constants(s) for s in range(2)]
    return dv0, th, base, rebuilds


def test_case_exercises_resorts_and_slip(adjoint):
    dv0, th, base, rebuilds = adjoint
    assert rebuilds > 5
    assert np.all(th[:, 3] != 0) and np.all(th[:, 4] != 0)   # friction was active


@pytest.mark.parametrize("i,c", [(0, 2), (5, 0), (33, 1), (70, 2), (99, 0)])
def test_initial_velocity_gradient_matches_fd(case, adjoint, i, c):
    dv0 = adjoint[0]
    v0 = case[4]
    h = 1e-6 * max(1.0, abs(v0[i, c]))
    vp, vm = v0.copy(), v0.copy()
    vp[i, c] += h
    vm[i, c] -= h
    fd = (loss(case, run(case, v=vp)) - loss(case, run(case, v=vm))) / (2 * h)
    assert abs(dv0[i, c] - fd) <= 1e-5 * abs(fd) + 1e-12, (dv0[i, c], fd)


@pytest.mark.parametrize("s", [0, 1])
@pytest.mark.parametrize("k,name", list(enumerate(["kn", "kt", "2beta", "mu", "mu_wall"])))
def test_law_constant_gradient_matches_fd(case, adjoint, s, k, name):
    th, base = adjoint[1], adjoint[2]
    h = 1e-6 * abs(base[s][k])
    cp = [b.copy() for b in base]
    cm = [b.copy() for b in base]
    cp[s][k] += h
    cm[s][k] -= h
    fd = (loss(case, run(case, consts=cp)) - loss(case, run(case, consts=cm))) / (2 * h)
    assert abs(th[s, k] - fd) <= 1e-5 * abs(fd) + 1e-12, (name, th[s, k], fd)


def test_windowed_adjoint_matches_fd_at_full_horizon():
    """The reverse sweep over the last 50 steps of a 3,000-step settling run
    (1,000 spheres of the calibration workload, FP64 restatement) against
    central finite differences of the same windowed problem (the law
    constants perturbed during the last 50 steps only; loss: mean height).

    Over the whole horizon the pathwise derivative is not usable: it grows
    about 5 % per step (the adjoint of the mean height with respect to the
    initial velocities is ~1e-3 after 100 steps, ~4e3 after 400, ~1e29
    after 1,600), and finite differences of the full run depend on the step
    (0.27, -0.05, 0.03 for h = 3e-3, 1e-2, 3e-2 at 1,600 steps): dense
    granular flow is chaotic.  Within a window the derivative is that of the
    branch the contacts took; the differences must stay below the
    perturbation that flips a contact onset or a stick/slip state (with
    ~3e5 such decisions in the window, h = 1e-6 flips one for kn here),
    and above the rounding noise (h = 1e-9 and below)."""
    N, T, WIN, H = 1000, 3000, 50, 1e-7
    S, W, p, r = calibrate.calibration_ensemble(nsys=1, n=N, seed=4)
    v0 = calibrate.initial_velocity(len(p))

    def fresh():
        o = EnsRestated(S, W, 1, 1e-5, 0.02, 32, precision="f64")
        o.set_state(p, r, v0)
        assert o.step(T - WIN) == 0
        return o

    o = fresh()
    c0 = o.constants(0)
    assert o.adj_record(WIN) == 0
    gx = np.zeros(p.shape)
    gx[:, 2] = 1.0 / N
    _, _, _, th = o.adj_reverse(gx, np.zeros(p.shape), np.zeros(p.shape))
    for k, name in ((0, "kn"), (2, "2 beta"), (3, "mu")):
        L = []
        for sgn in (1.0, -1.0):
            q = fresh()
            c = c0.copy()
            c[k] *= 1.0 + sgn * H
            q.set_constants(0, c)
            q.step(WIN)
            L.append(q.state()["pos"][:, 2].mean())
        fd = (L[0] - L[1]) / (2.0 * H * c0[k])
        rel = abs(fd - th[0][k]) / abs(fd)
        print("%s: windowed adjoint %.6e, central FD %.6e, relative %.1e" % (name, th[0][k], fd, rel))
        assert rel < 1e-3, (name, fd, th[0][k])
