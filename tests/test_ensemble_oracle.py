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


def _closest_on_triangles(p, tri):
    """Closest points of triangles tri (m, 3, 3) to points p (n, 3), FP64,
    by Voronoi regions (Ericson, Real-Time Collision Detection, 5.1.5)."""
    a, b, c = tri[None, :, 0], tri[None, :, 1], tri[None, :, 2]
    p = p[:, None]
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = (ab * ap).sum(-1), (ac * ap).sum(-1)
    bp, cp = p - b, p - c
    d3, d4 = (ab * bp).sum(-1), (ac * bp).sum(-1)
    d5, d6 = (ab * cp).sum(-1), (ac * cp).sum(-1)
    va, vb, vc = d3 * d6 - d5 * d4, d5 * d2 - d1 * d6, d1 * d4 - d3 * d2
    with np.errstate(divide="ignore", invalid="ignore"):
        den = 1.0 / (va + vb + vc)
        q = a + ab * (vb * den)[..., None] + ac * (vc * den)[..., None]
        e_ab = a + ab * (d1 / (d1 - d3))[..., None]
        e_ac = a + ac * (d2 / (d2 - d6))[..., None]
        e_bc = b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)))[..., None]
    q = np.where(((va <= 0) & (d4 - d3 >= 0) & (d5 - d6 >= 0))[..., None], e_bc, q)
    q = np.where(((vb <= 0) & (d2 >= 0) & (d6 <= 0))[..., None], e_ac, q)
    q = np.where(((d6 >= 0) & (d5 <= d6))[..., None], c + 0 * q, q)
    q = np.where(((vc <= 0) & (d1 >= 0) & (d3 <= 0))[..., None], e_ab, q)
    q = np.where(((d3 >= 0) & (d4 <= d3))[..., None], b + 0 * q, q)
    q = np.where(((d1 <= 0) & (d2 <= 0))[..., None], a + 0 * q, q)
    return q


def _onset_particles(S, walls, pos, rad, band=3e-7):
    """Particles with a contact (pair or wall) whose overlap is within
    band * (radius sum) of zero, a few FP32 rounding steps: whether FP32 and
    FP64 count such a contact depends on the rounding of the contact test,
    and the damped normal force jumps at contact onset, so their forces are
    not a measure of the law's arithmetic."""
    pos = pos.astype(np.float64)
    rad = rad.astype(np.float64)
    out = np.zeros(len(pos), bool)
    lo = 0
    for s in S:
        hi = lo + s.n
        P, R = pos[lo:hi], rad[lo:hi]
        d = np.linalg.norm(P[:, None] - P[None], axis=2)
        sr = R[:, None] + R[None]
        amb = np.abs(d - sr) < band * sr
        np.fill_diagonal(amb, False)
        out[lo:hi] |= amb.any(axis=1)
        for w in list(walls[s.wall0:s.wall0 + s.nwalls]):
            q = np.array(w.p, np.float64)
            if w.kind == E.WALL_PLANE:
                dist = P @ q[:3] - q[3]
            else:
                v = P - q[:3]
                rv = v - np.outer(v @ q[3:6], q[3:6])
                dist = q[6] - np.linalg.norm(rv, axis=1)
            out[lo:hi] |= np.abs(dist - R) < band * R
        if s.ntris:
            tri = np.array([list(w.p)[:9] for w in walls[s.tri0:s.tri0 + s.ntris]],
                           np.float64).reshape(-1, 3, 3)
            q = _closest_on_triangles(P, tri)
            dist = np.linalg.norm(P[:, None] - q, axis=2)
            out[lo:hi] |= (np.abs(dist - R[:, None]) < band * R[:, None]).any(axis=1)
        lo = hi
    return out


def _fp32_force_error(S, W, pos, rad, vel, avel, law, dt=1e-5):
    """One step's contact forces and torques in FP32 against FP64 from the
    same state (caller's order), as fractions of the largest FP64 force and
    torque, over the particles with no contact at its onset."""
    out = {}
    for prec in ("f32", "f64"):
        o, _ = run(S, W, pos, rad, vel=vel, avel=avel, law=law, dt=dt, steps=1, prec=prec)
        f, t = o.forces()
        order = np.argsort(o.state()["pid"])
        out[prec] = (f[order], t[order])
    keep = ~_onset_particles(S, W, pos, rad)
    (f32, t32), (f64, t64) = out["f32"], out["f64"]
    ef = np.abs(f32 - f64)[keep].max() / np.abs(f64).max()
    et = np.abs(t32 - t64)[keep].max() / np.abs(t64).max()
    return ef, et, int((~keep).sum())


@pytest.mark.parametrize("law", [E.LAW_LINEAR, E.LAW_HERTZ_MINDLIN])
def test_box_settles_fp32_error_stated(law):
    """Two box systems (plane walls) settle for 2500 steps (FP32, bounded
    state); from that state one step runs in FP32 and in FP64, for the linear
    and the Hertz-Mindlin law with tangential history and rolling friction.
    The FP32 force error -- the error the product inherits -- is below 1e-5
    of the largest force: the overlaps cancel their large terms exactly
    (accurate overlaps, csrc/ens_kernels.cuh)."""
    S, W, p, r = synth.box_ensemble([500, 900], seed=2, mus=[0.3, 0.7], restitutions=[0.4, 0.8])
    o, st = run(S, W, p, r, dt=1e-5, steps=2500, prec="f32", skin=0.02)
    assert st == 0
    s = o.state()
    assert np.abs(s["vel"]).max() < 100.0
    order = np.argsort(s["pid"])
    for sy in S:
        sy.youngs, sy.mu_roll = 2e5, 0.02
    ef, et, nex = _fp32_force_error(S, W, s["pos"][order], s["radius"][order], s["vel"][order],
                                    s["avel"][order], law)
    print("box, law %d: FP32 vs FP64 after one step: force %.2e, torque %.2e of the largest "
          "(%d particles at contact onset left out)" % (law, ef, et, nex))
    assert ef < 1e-5 and et < 1e-5, (ef, et)


def funnel_triangles(r_in, r_out, z_in, z_out, n_seg=12, n_ring=3):
    """A truncated cone (funnel) from radius r_in at z_in to r_out at z_out,
    axis z, as n_seg x n_ring quads of two triangles each."""
    tris = []
    rs = np.linspace(r_in, r_out, n_ring + 1)
    zs = np.linspace(z_in, z_out, n_ring + 1)
    ang = np.linspace(0.0, 2 * np.pi, n_seg + 1)
    for k in range(n_ring):
        for j in range(n_seg):
            q = [(rs[k + dk] * np.cos(ang[j + dj]), rs[k + dk] * np.sin(ang[j + dj]), zs[k + dk])
                 for dk, dj in ((0, 0), (1, 0), (1, 1), (0, 1))]
            tris.append(E.triangle(q[0], q[1], q[2]))
            tris.append(E.triangle(q[0], q[2], q[3]))
    return tris


@pytest.fixture(scope="module")
def funnel_bed():
    """300 spheres settled for 12,000 steps in a cylinder (r = 1.5 cm, axis
    z) over a 45-degree funnel of 72 triangles down to a plane floor."""
    rng = np.random.default_rng(5)
    n = 300
    walls = [E.cylinder((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 1.5), E.plane((0.0, 0.0, 1.0), 0.0)]
    tris = funnel_triangles(0.4, 1.6, 0.0, 1.2)
    walls += tris
    S = [free_system(n, E.LAW_LINEAR, L=16.0, cell=0.5, gravity=(0.0, 0.0, -981.0), walls=(0, 2),
                     tris=(2, len(tris)), youngs=2e5, mu_roll=0.02)]
    g = np.arange(-1.26, 1.27, 0.42)
    gx, gy, gz = np.meshgrid(g, g, 1.4 + 0.42 * np.arange(20), indexing="ij")
    lat = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1)
    lat = lat[np.hypot(lat[:, 0], lat[:, 1]) < 1.25]
    pos = lat[np.lexsort((lat[:, 0], lat[:, 1], lat[:, 2]))][:n]
    pos = pos + rng.uniform(-0.02, 0.02, pos.shape)
    rad = rng.uniform(0.1, 0.2, n)
    o, st = run(S, walls, pos, rad, law=E.LAW_LINEAR, dt=1e-5, steps=12000, prec="f32", skin=0.02)
    assert st == 0
    s = o.state()
    order = np.argsort(s["pid"])
    tri = np.array([list(w.p)[:9] for w in tris], np.float64).reshape(-1, 3, 3)
    q = _closest_on_triangles(s["pos"], tri)
    on_funnel = (np.linalg.norm(s["pos"][:, None] - q, axis=2) < s["radius"][:, None]).any(axis=1)
    on_wall = np.hypot(s["pos"][:, 0], s["pos"][:, 1]) + s["radius"] > 1.5
    assert on_funnel.sum() > 20 and on_wall.sum() > 1, (on_funnel.sum(), on_wall.sum())
    return S, walls, {k: s[k][order] for k in ("pos", "radius", "vel", "avel")}


@pytest.mark.parametrize("law", [E.LAW_LINEAR, E.LAW_HERTZ_MINDLIN])
def test_cylinder_and_triangles_fp32_error_stated(funnel_bed, law):
    """On the settled funnel bed (face, edge and vertex contacts with the
    triangles, the cylinder, the floor), one step's FP32 contact forces
    against FP64 from the same state: below 1e-5 of the largest force for
    both laws."""
    S, walls, b = funnel_bed
    for sy in S:
        sy.youngs, sy.mu_roll = 2e5, 0.02
    ef, et, nex = _fp32_force_error(S, walls, b["pos"], b["radius"], b["vel"], b["avel"], law)
    print("cylinder + funnel triangles, law %d: FP32 vs FP64 after one step: force %.2e, torque "
          "%.2e of the largest (%d particles at contact onset left out)" % (law, ef, et, nex))
    assert ef < 1e-5 and et < 1e-5, (ef, et)
