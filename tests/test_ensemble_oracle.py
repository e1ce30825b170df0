"""The ensemble restatement (oracle/ens_oracle.c) against closed-form
mechanics: these are the pins of the extended contact laws, which the
reference does not have (its law is Collision_Response.cuh:374-494).

Each case runs the FP64 build unless it says otherwise; the tolerances are
stated per case and come from the time step (a contact lasts ~20-60 steps
here) and from the damping model.
"""
import math

import numpy as np
import pytest

from bindings import EnsRestated
from blaze import ensemble as E
from blaze import synth

RHO = 2500e-6  # kg/cm^3


def free_system(n, law=E.LAW_LINEAR, L=20.0, cell=1.0, gravity=(0.0, 0.0, 0.0), e=0.5, mu=0.4,
                mu_roll=0.0, kn=1e5, youngs=1e5, walls=(0, 0), tris=(0, 0)):
    s = E.System()
    s.n = n
    for k in range(3):
        s.origin[k] = -L / 2
        s.ncells[k] = int(L / cell)
        s.gravity[k] = gravity[k]
    s.cell = cell
    s.density = RHO
    s.kn, s.kt_ratio, s.youngs, s.poisson = kn, 2.0 / 7.0, youngs, 0.3
    s.restitution, s.mu, s.mu_wall, s.mu_roll = e, mu, mu, mu_roll
    s.wall0, s.nwalls = walls
    s.tri0, s.ntris = tris
    return s


def run(systems, walls, pos, rad, vel=None, avel=None, law=E.LAW_LINEAR, dt=1e-6, steps=1,
        prec="f64", skin=0.05):
    o = EnsRestated(systems, walls, law, dt, skin, 32, precision=prec)
    o.set_state(pos, rad, vel, avel)
    st = o.step(steps)
    return o, st


@pytest.mark.parametrize("law", [E.LAW_LINEAR, E.LAW_HERTZ_MINDLIN])
def test_pair_forces_are_exact_negatives(law):
    """Newton's third law bit for bit in FP32: the (j, i) evaluation of a
    contact is the exact negation of (i, j), spin, sliding and rolling
    friction included."""
    rng = np.random.default_rng(7)
    for trial in range(20):
        r = rng.uniform(0.1, 0.2, size=2)
        d = (r[0] + r[1]) * rng.uniform(0.97, 0.999)
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        pos = np.array([[0.0, 0.0, 0.0], d * u])
        vel = rng.normal(scale=20.0, size=(2, 3))
        avel = rng.normal(scale=300.0, size=(2, 3))
        S = [free_system(2, law, mu_roll=0.05)]
        o, st = run(S, [], pos, r, vel, avel, law=law, dt=1e-6, steps=3, prec="f32")
        assert st == 0
        f, _ = o.forces()
        assert np.any(f != 0)
        np.testing.assert_array_equal(f[0], -f[1])


@pytest.mark.parametrize("law,e", [(E.LAW_LINEAR, 0.5), (E.LAW_LINEAR, 0.8),
                                   (E.LAW_HERTZ_MINDLIN, 0.6)])
def test_head_on_restitution(law, e):
    """Two equal spheres, head on, no gravity: the separation speed over the
    approach speed equals the restitution the damping was derived from
    (linear: exact in continuous time, 2 %; Hertz-Mindlin with the
    2 sqrt(5/6) beta damping: an approximation, 6 %), at dt = 1e-7 s."""
    r = 0.15
    pos = np.array([[-0.151, 0.0, 0.0], [0.151, 0.0, 0.0]])
    v0 = 50.0
    vel = np.array([[v0, 0.0, 0.0], [-v0, 0.0, 0.0]])
    S = [free_system(2, law, e=e, kn=1e5, youngs=1e5)]
    o, st = run(S, [], pos, np.array([r, r]), vel, law=law, dt=1e-7, steps=3000)
    assert st == 0
    s = o.state()
    order = np.argsort(s["pid"])
    v = s["vel"][order]
    ratio = (v[1, 0] - v[0, 0]) / (2 * v0)
    tol = 0.02 if law == E.LAW_LINEAR else 0.06
    assert abs(ratio - e) < tol * e, ratio


def floor_case(tri=False):
    """One sphere on the plane z = 0 (or on two triangles covering it)."""
    if tri:
        walls = [E.triangle((-5, -5, 0), (5, -5, 0), (5, 5, 0)),
                 E.triangle((-5, -5, 0), (5, 5, 0), (-5, 5, 0))]
        S = [free_system(1, gravity=(0, 0, -981.0), mu=0.4, tris=(0, 2))]
    else:
        walls = [E.plane((0, 0, 1), 0.0)]
        S = [free_system(1, gravity=(0, 0, -981.0), mu=0.4, walls=(0, 1))]
    return S, walls


@pytest.mark.parametrize("tri", [False, True])
def test_sliding_sphere_ends_rolling_at_five_sevenths(tri):
    """A sphere launched sliding (no spin) on a floor with Coulomb friction
    decelerates at mu g until it rolls; a solid sphere then keeps 5/7 of the
    launch speed.  Within 1 % (the normal spring's settling wiggle)."""
    S, walls = floor_case(tri)
    r = 0.15
    m = RHO * 4 / 3 * math.pi * r ** 3
    z0 = r - m * 981.0 / 1e5  # resting overlap of the linear spring
    v0 = 30.0
    o, st = run(S, walls, np.array([[0.0, 0.0, z0]]), np.array([r]),
                np.array([[v0, 0.0, 0.0]]), dt=1e-5, steps=4000)
    assert st == 0
    s = o.state()
    assert abs(s["vel"][0, 0] / v0 - 5.0 / 7.0) < 0.01, s["vel"][0, 0] / v0
    # rolling: contact-point speed v - w x r ~ 0
    assert abs(s["vel"][0, 0] - s["avel"][0, 1] * r) < 0.01 * v0


def test_triangle_floor_matches_plane_floor():
    """Face contacts with a triangle mesh give the plane's contact (FP64,
    1e-9 relative over 2000 steps of sliding into rolling)."""
    r = 0.15
    st0 = (np.array([[0.3, -0.2, r - 0.0005]]), np.array([r]), np.array([[25.0, 5.0, 0.0]]))
    out = []
    for tri in (False, True):
        S, walls = floor_case(tri)
        o, st = run(S, walls, *st0, dt=1e-5, steps=2000)
        assert st == 0
        out.append(o.state())
    np.testing.assert_allclose(out[1]["pos"], out[0]["pos"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(out[1]["vel"], out[0]["vel"], rtol=1e-9, atol=1e-9)


def test_rolling_friction_decelerates_at_five_sevenths_mu_r_g():
    """Constant rolling torque mu_r f_n R on a rolling sphere: deceleration
    (5/7) mu_r g for a solid sphere.  Within 3 %."""
    r = 0.15
    mu_r = 0.05
    S = [free_system(1, gravity=(0, 0, -981.0), mu=0.5, mu_roll=mu_r, walls=(0, 1))]
    walls = [E.plane((0, 0, 1), 0.0)]
    m = RHO * 4 / 3 * math.pi * r ** 3
    z0 = r - m * 981.0 / 1e5
    v0 = 20.0
    T = 0.5
    o, st = run(S, walls, np.array([[0.0, 0.0, z0]]), np.array([r]), np.array([[v0, 0.0, 0.0]]),
                np.array([[0.0, v0 / r, 0.0]]), dt=1e-5, steps=int(T / 1e-5))
    assert st == 0
    v = o.state()["vel"][0, 0]
    decel = (v0 - v) / T
    expect = 5.0 / 7.0 * mu_r * 981.0
    assert abs(decel / expect - 1.0) < 0.03, (decel, expect)


def test_cylinder_holds_particles_inside():
    """A cylinder wall (axis z) keeps a spray of spheres inside its radius."""
    rng = np.random.default_rng(3)
    n = 200
    walls = [E.cylinder((0, 0, 0), (0, 0, 1), 2.0), E.plane((0, 0, 1), -5.0)]
    S = [free_system(n, gravity=(0, 0, -981.0), walls=(0, 2), L=14.0, cell=0.5)]
    ang = rng.uniform(0, 2 * np.pi, n)
    rr = rng.uniform(0, 1.5, n)
    pos = np.stack([rr * np.cos(ang), rr * np.sin(ang), rng.uniform(-4.5, 4.5, n)], 1)
    vel = rng.normal(scale=40.0, size=(n, 3))
    o, st = run(S, walls, pos, np.full(n, 0.1), vel, dt=1e-5, steps=3000, skin=0.05)
    s = o.state()
    rho = np.hypot(s["pos"][:, 0], s["pos"][:, 1])
    assert rho.max() < 2.0 - 0.1 + 0.02, rho.max()


def test_box_settles_fp32_error_stated():
    """Two box systems settle for 2500 steps (FP32, bounded state); from the
    settled state one step runs in FP32 and in FP64, and the FP32 contact
    force error -- the error the product inherits -- is stated and bounded."""
    S, W, p, r = synth.box_ensemble([500, 900], seed=2, mus=[0.3, 0.7], restitutions=[0.4, 0.8])
    o, st = run(S, W, p, r, dt=1e-5, steps=2500, prec="f32", skin=0.02)
    assert st == 0
    s = o.state()
    assert np.abs(s["vel"]).max() < 100.0
    # settled state in the caller's order (system-concatenated), as set_state wants it
    order = np.argsort(s["pid"])
    args = (s["pos"][order], s["radius"][order], s["vel"][order], s["avel"][order])
    o32, _ = run(S, W, *args[:2], vel=args[2], avel=args[3], dt=1e-5, steps=1, prec="f32")
    o64, _ = run(S, W, *args[:2], vel=args[2], avel=args[3], dt=1e-5, steps=1, prec="f64")
    f32, _ = o32.forces()
    f64, _ = o64.forces()
    scale = np.abs(f64).max()
    assert scale > 0
    err = np.abs(f32 - f64).max() / scale
    # The overlap (ra + rb) - |xa - xb| cancels in FP32: at overlaps of
    # ~1e-5 cm between spheres of ~0.3 cm the distance carries ~3e-8 cm of
    # rounding, i.e. ~1e-3 of the overlap and of the normal force of the
    # lightest contacts.  Measured here: 6e-4 of the largest force.
    print("FP32 vs FP64 contact force after one step: max %.2e of the largest force" % err)
    assert err < 2e-3
