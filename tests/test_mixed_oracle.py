"""Mixed charge (spheres and convex polyhedra) on the CPU: the shapes' mass
properties (the library's host function) against closed forms, the rock
generator, and the FP64 restatement (oracle/ens_oracle.c) against
mechanics with known answers:
  - a cube resting on the floor: contact force = weight, overlap = m g / kn,
    no turn;
  - a sphere resting on a cube's face: force along the face normal;
  - two cubes face on face and two cubes with crossing edges (each turned
    45 degrees, about x and about y): the contact normal is the face normal /
    the cross product of the edges, the force kn delta, no torque;
  - a loose cluster of rocks and balls without gravity or walls: the
    contact forces sum to zero (Newton's third law) at every step, and
    without damping and friction the kinetic energy after the collisions
    returns to its value before them.
"""
import math

import numpy as np
import pytest

from bindings import EnsRestated
from blaze import ensemble as E
from blaze import synth


def hull_shape(v, density):
    from scipy.spatial import ConvexHull
    v = np.asarray(v, np.float64)
    h = ConvexHull(v)
    f = h.simplices.copy()
    c = v.mean(axis=0)
    for k in range(len(f)):
        a, b, cc = v[f[k]]
        if np.dot(np.cross(b - a, cc - a), a - c) < 0:
            f[k] = f[k][[0, 2, 1]]
    return E.shape(v, f, density), f


CUBE = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)])
RHO = 2.7e-3   # kg/cm^3


def test_mass_properties_closed_forms():
    a = 2.0
    s, _ = hull_shape(CUBE * a, 1e-3)
    m, com, J, rb = E.mass_properties(s)
    m0 = float(np.float32(1e-3)) * a ** 3
    assert abs(m - m0) < 1e-12 * m0
    np.testing.assert_allclose(J, np.eye(3) * m0 * a * a / 6.0, rtol=1e-12, atol=1e-15)
    assert np.abs(com).max() < 1e-15
    assert abs(rb - math.sqrt(3.0)) < 2e-7 and rb >= math.sqrt(3.0) * (1 - 1e-7)
    # regular tetrahedron of edge 2 sqrt 2: I = m a^2 / 20 about any axis
    t = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], np.float64)
    s, _ = hull_shape(t, 1e-3)
    m, com, J, rb = E.mass_properties(s)
    m0 = float(np.float32(1e-3)) * 8.0 / 3.0
    assert abs(m - m0) < 1e-12 * m0
    np.testing.assert_allclose(J, np.eye(3) * m0 * 8.0 / 20.0, rtol=1e-12, atol=1e-15)


def test_invalid_shapes_rejected():
    s, f = hull_shape(CUBE, RHO)
    bad = E.shape(CUBE, f[:, [0, 2, 1]], RHO)        # faces turned inside out
    with pytest.raises(Exception):
        E.mass_properties(bad)
    dent = CUBE.copy()
    dent[0] *= 0.3                                   # a vertex pushed in: not convex
    bad = E.shape(dent, f, RHO)
    with pytest.raises(Exception):
        E.mass_properties(bad)
    bad = E.shape(CUBE, f[:-1], RHO)                 # open
    with pytest.raises(Exception):
        E.mass_properties(bad)


def test_rock_generator():
    rng = np.random.default_rng(2)
    for _ in range(40):
        v, f = synth.rock_hull(rng)
        assert 8 <= len(v) <= 16 and len(f) == 2 * len(v) - 4
        # points on a sphere of radius <= 1 cm, moved to their centre of mass
        r = np.linalg.norm(v, axis=1)
        assert 0.25 <= r.max() <= 1.25
        s = E.shape(v, f, RHO)
        m, com, J, rb = E.mass_properties(s)
        assert np.abs(com).max() < 1e-6 * rb
        assert np.all(np.linalg.eigvalsh(J) > 0)


def scene(pos, rad, shapes, shape_of, quat, L=20.0, gravity=(0.0, 0.0, -981.0), kn=1e5,
          restitution=0.4, mu=0.6, dt=1e-5, precision="f64", vel=None, avel=None):
    rb = max([max(rad)] + [float(np.linalg.norm(np.asarray(s.verts).reshape(-1, 3)[:s.nverts],
                                                axis=1).max()) for s in shapes])
    cell = 2.0 * rb + 0.04 + 1e-3
    walls = synth.box_walls(L, L)
    s = synth.box_system(len(pos), L, L, cell, 0, density=7.8e-3, kn=kn, restitution=restitution,
                         mu=mu, gravity=gravity)
    o = EnsRestated([s], walls, E.LAW_LINEAR, dt, 0.04, 32, precision=precision)
    o.set_state(np.asarray(pos, np.float64), np.asarray(rad, np.float64), vel, avel)
    o.set_polyhedra(shapes, np.asarray(shape_of, np.int32), np.asarray(quat, np.float64))
    return o, s


def quat_about(axis, ang):
    a = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    return np.concatenate([[math.cos(ang / 2)], a * math.sin(ang / 2)])


def test_cube_rests_on_the_floor():
    cube, _ = hull_shape(CUBE, RHO)
    m = E.mass_properties(cube)[0]
    o, _ = scene([[10.0, 10.0, 0.5]], [0.87], [cube], [0], [[1, 0, 0, 0]])
    o.step(30000)
    f, t = o.forces()
    st = o.state()
    q = o.orientations()
    delta = m * 981.0 / 1e5
    print("cube on the floor: force %s (weight %.6g), sink %.4g (m g / kn %.4g)"
          % (f[0], m * 981.0, 0.5 - st["pos"][0, 2], delta))
    assert abs(f[0, 2] - m * 981.0) < 1e-3 * m * 981.0
    assert np.abs(f[0, :2]).max() < 1e-9 * m * 981.0
    assert abs((0.5 - st["pos"][0, 2]) - delta) < 1e-3 * delta
    assert np.abs(st["avel"][0]).max() < 1e-9 and np.abs(q[0] - [1, 0, 0, 0]).max() < 1e-12
    assert st["status"] == 0


def test_sphere_rests_on_a_face():
    cube, _ = hull_shape(CUBE, RHO)
    r = 0.3
    o, s = scene([[10.0, 10.0, 0.5], [10.1, 10.05, 1.0 + r]], [0.87, r], [cube], [0, -1],
                 [[1, 0, 0, 0], [1, 0, 0, 0]])
    o.step(30000)
    f, t = o.forces()
    st = o.state()
    ms = s.density * 4.0 / 3.0 * math.pi * r ** 3
    i = int(np.nonzero(st["pid"] == 1)[0][0])
    print("sphere on a cube: force on the sphere %s (weight %.6g)" % (f[i], ms * 981.0))
    assert abs(f[i, 2] - ms * 981.0) < 1e-3 * ms * 981.0
    # under the off-centre load the cube tilts by ~4 delta x / side^2 (the
    # depth-weighted contact point moves under the load): 1e-5 rad here
    assert np.abs(f[i, :2]).max() < 1e-4 * ms * 981.0
    # it settles where it was put (a slide of ~1e-4 cm while the cube tilts)
    assert np.abs(st["pos"][i, :2] - [10.1, 10.05]).max() < 1e-3
    assert np.abs(st["vel"]).max() < 1e-3


@pytest.mark.parametrize("kind", ["face", "edge"])
def test_cube_pair_normal_and_force(kind):
    cube, _ = hull_shape(CUBE, RHO)
    delta = 2e-4
    if kind == "face":
        qa, qb = [1, 0, 0, 0], [1, 0, 0, 0]
        gap = 1.0
    else:   # A turned 45 degrees about x (top edge along x), B about y (bottom edge along y)
        qa, qb = quat_about([1, 0, 0], math.pi / 4), quat_about([0, 1, 0], math.pi / 4)
        gap = math.sqrt(2.0)
    z0 = 10.0
    o, _ = scene([[10.0, 10.0, z0], [10.0, 10.0, z0 + gap - delta]], [0.87, 0.87], [cube], [0, 0],
                 [qa, qb], gravity=(0.0, 0.0, 0.0))
    o.step(1)
    f, t = o.forces()
    st = o.state()
    ib = int(np.nonzero(st["pid"] == 1)[0][0])
    ia = 1 - ib
    d_true = gap - ((z0 + gap - delta) - z0)   # the FP64 restatement keeps the inputs exact
    print("%s contact: force on B %s, kn delta %.6g, torque on B %s"
          % (kind, f[ib], 1e5 * d_true, t[ib]))
    np.testing.assert_allclose(f[ib], [0.0, 0.0, 1e5 * d_true], rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(f[ia], -f[ib], rtol=0, atol=1e-12)
    # no lever arm (the turns are the float-rounded 45 degrees)
    tol = 1e-6 * np.linalg.norm(f[ib]) * 1.0
    assert np.abs(t[ib]).max() < tol and np.abs(t[ia]).max() < tol


def cluster(seed=5, n_rocks=8, n_spheres=40):
    rng = np.random.default_rng(seed)
    shapes = synth.rock_shapes(n_rocks, seed=seed)
    pts = synth.lattice_fill(None, (8.0, 8.0, 8.0), (12.5, 12.5, 12.5), 1.55, rng)
    pts = pts[rng.permutation(len(pts))[:n_rocks + n_spheres]]
    rad = np.concatenate([rng.uniform(0.3, 0.6, n_spheres),
                          [synth._bounding_radius(s) for s in shapes]])
    so = np.concatenate([np.full(n_spheres, -1), np.arange(n_rocks)])
    q = np.zeros((len(pts), 4))
    q[:, 0] = 1.0
    q[n_spheres:] = synth.random_quaternions(rng, n_rocks)
    centre = np.array([10.25, 10.25, 10.25])
    vel = (centre - pts) * 20.0 + rng.normal(scale=5.0, size=pts.shape)   # inward
    avel = np.zeros_like(pts)
    avel[n_spheres:] = rng.normal(scale=20.0, size=(n_rocks, 3))
    return pts, rad, shapes, so, q, vel, avel


def test_third_law_in_a_cluster():
    pts, rad, shapes, so, q, vel, avel = cluster()
    o, _ = scene(pts, rad, shapes, so, q, gravity=(0.0, 0.0, 0.0), L=40.0, vel=vel, avel=avel)
    worst, contacts = 0.0, 0
    for k in range(300):
        o.step(10)
        f, t = o.forces()
        nz = np.linalg.norm(f, axis=1) > 0
        contacts = max(contacts, int(nz.sum()))
        if nz.any():
            worst = max(worst, np.linalg.norm(f.sum(axis=0)) / np.linalg.norm(f, axis=1).max())
    print("cluster: up to %d particles in contact; |sum F| / max |F| = %.2e" % (contacts, worst))
    assert contacts >= 10
    assert worst < 1e-12


def kinetic_energy(o, shapes, so, rho_s):
    st = o.state()
    q = o.orientations()
    e = 0.0
    for k in range(len(st["pid"])):
        pid = st["pid"][k]
        v, w = st["vel"][k], st["avel"][k]
        if so[pid] < 0:
            m = rho_s * 4.0 / 3.0 * math.pi * st["radius"][k] ** 3
            e += 0.5 * m * v @ v + 0.5 * (0.4 * m * st["radius"][k] ** 2) * w @ w
        else:
            m, _, J, _ = E.mass_properties(shapes[so[pid]])
            qw, qx, qy, qz = q[k]
            R = np.array([[1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy)],
                          [2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx)],
                          [2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)]])
            wb = R.T @ w
            e += 0.5 * m * v @ v + 0.5 * wb @ J @ wb
    return e


def test_elastic_frictionless_collisions_keep_energy():
    """Restitution 1 (no damping), no friction: two rocks and a ball meet
    and part; the kinetic energy afterwards equals the energy before within
    the integrator's error."""
    shapes = synth.rock_shapes(2, seed=7)
    pts = np.array([[9.0, 10.0, 10.0], [11.0, 10.1, 10.05], [10.0, 11.2, 10.0]])
    rad = np.array([synth._bounding_radius(shapes[0]), synth._bounding_radius(shapes[1]), 0.4])
    so = np.array([0, 1, -1])
    q = np.array([quat_about([1, 2, 3], 0.7), quat_about([3, -1, 2], 1.9), [1, 0, 0, 0]])
    vel = np.array([[50.0, 0.0, 0.0], [-50.0, 0.0, 0.0], [0.0, -40.0, 0.0]])
    avel = np.array([[0.0, 0.0, 30.0], [10.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    o, s = scene(pts, rad, shapes, so, q, gravity=(0.0, 0.0, 0.0), L=40.0, restitution=1.0,
                 mu=0.0, dt=2e-6, vel=vel, avel=avel)
    e0 = kinetic_energy(o, shapes, so, s.density)
    touched = False
    for _ in range(100):
        o.step(200)
        f, _ = o.forces()
        touched = touched or bool(np.abs(f).max() > 0)
    f, _ = o.forces()
    e1 = kinetic_energy(o, shapes, so, s.density)
    print("elastic collisions: E before %.6g after %.6g (relative change %.2e), touched %s"
          % (e0, e1, e1 / e0 - 1.0, touched))
    assert touched and np.abs(f).max() == 0.0
    assert abs(e1 / e0 - 1.0) < 2e-3


def test_mixed_charge_generators():
    """The mixed charges start without overlaps: every ball keeps 0.02 cm
    from every rock's bounding sphere and from the other balls, rocks from
    each other; the mill's charge holds the configuration's 20 : 1 count
    ratio inside the lifter ring."""
    from scipy.spatial import cKDTree
    cases = [synth.mixed_box_ensemble(),
             synth.mill_mixed_ensemble(n_spheres=20000, n_rocks=1000)]
    for S, W, p, r, sh, so, q in cases:
        p = p.astype(np.float64)
        rk, sp = so >= 0, so < 0
        d, k = cKDTree(p[rk]).query(p[sp])
        assert np.all(d - r[sp] - r[rk][k] >= 0.02 - 1e-5)
        pairs = cKDTree(p).query_pairs(2.5, output_type="ndarray")
        gap = np.linalg.norm(p[pairs[:, 0]] - p[pairs[:, 1]], axis=1) - r[pairs[:, 0]] - r[pairs[:, 1]]
        assert gap.min() > 0.0
        assert np.all(2 * r + 0.04 <= S[0].cell)
        np.testing.assert_allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-6)
    S, W, p, r, sh, so, q = cases[1]
    assert (so < 0).sum() == 20 * (so >= 0).sum()
    assert np.hypot(p[:, 0], p[:, 1]).max() < 50.0 - 4.0


@pytest.mark.parametrize("case", ["mixed_drum", "sphere_drum"])
def test_restatement_triangle_lists_change_nothing(case):
    """The restatement's per-cell triangle candidates give the same run, bit
    for bit, as testing every triangle of the system: 400 steps from the
    state after 12,000 (the charge on the liner and lifters)."""
    kw = dict(R=12.0, L=8.0, n_seg=48, n_len=6, n_lifters=4, lifter_w=2.0, lifter_h=2.0, kn=1e5)
    if case == "mixed_drum":
        S, W, p, r, sh, so, q = synth.mill_mixed_ensemble(n_spheres=400, n_rocks=24, **kw)
    else:
        S, W, p, r = synth.drum_mesh_ensemble(n=600, **kw)
        sh = None

    def restated(on, pos, vel=None, avel=None, quat=None):
        o = EnsRestated(S, W, E.LAW_LINEAR, 1e-5, 0.04, 32, precision="f32")
        o.use_tri_lists(on)
        o.set_state(pos, r, vel, avel)
        if sh is not None:
            o.set_polyhedra(sh, so, quat)
        return o

    o = restated(1, p, quat=None if sh is None else q)
    o.step(12000)
    st = o.state()
    qq = o.orientations()
    o.close()
    k = np.argsort(st["pid"])
    pos, vel, avel, quat = st["pos"][k], st["vel"][k], st["avel"][k], qq[k]
    reach = np.hypot(pos[:, 0], pos[:, 1]) + r
    assert reach.max() > 12.0 * np.cos(np.pi / 48) - 0.05      # touching the liner
    runs = []
    for on in (1, 0):
        o = restated(on, pos, vel, avel, quat)
        o.step(400)
        st = o.state()
        runs.append((st["pos"], st["vel"], st["avel"], st["status"]))
        o.close()
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a, b)


# ------------------------------------------------- narrow phases, brute force
def _rot(q):
    """The rotation of (w, x, y, z) as the restatement forms it: the FP32
    quaternion, normalised in FP64 through 2 / |q|^2."""
    q = [float(v) for v in q]
    qn = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    w, x, y, z = (float(np.float32(v / qn)) for v in q)
    s = 2.0 / (((w * w + x * x) + y * y) + z * z)
    return np.array([[1 - s * (y * y + z * z), s * (x * y - w * z), s * (x * z + w * y)],
                     [s * (x * y + w * z), 1 - s * (x * x + z * z), s * (y * z - w * x)],
                     [s * (x * z - w * y), s * (y * z + w * x), 1 - s * (x * x + y * y)]])


def _world(shape, q, centre):
    v = np.asarray(shape.verts, np.float64).reshape(-1, 3)[:shape.nverts]
    f = np.asarray(shape.faces).reshape(-1, 3)[:shape.nfaces]
    return v @ _rot(q).T + centre, f


def _axes(v, f):
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    e = set()
    for t in f:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            e.add((min(a, b), max(a, b)))
    return n, np.array([v[b] - v[a] for a, b in e])


def _penetration(va, fa, vb, fb):
    """Minimum overlap of two convex hulls over every face normal and every
    edge-pair cross product (full support extents, no pruning): their
    penetration depth when positive, a separation when negative."""
    na, ea = _axes(va, fa)
    nb, eb = _axes(vb, fb)
    cr = np.cross(ea[:, None, :], eb[None, :, :]).reshape(-1, 3)
    ln = np.linalg.norm(cr, axis=1)
    ax = np.concatenate([na, nb, cr[ln > 1e-9] / ln[ln > 1e-9, None]])
    pa, pb = va @ ax.T, vb @ ax.T
    over = np.minimum(pa.max(0) - pb.min(0), pb.max(0) - pa.min(0))
    return over.min()


def test_hull_pairs_against_brute_force():
    """Two rocks at random orientations and distances: the restatement's
    contact exists exactly when the brute-force separating-axis test finds
    overlap on every axis, and its depth (|F| / kn from rest) lies between
    the penetration depth and the depth over the feature tolerances (a face
    is kept over an edge pair up to 1 / 0.9 of its depth)."""
    rng = np.random.default_rng(11)
    shapes = synth.rock_shapes(12, seed=11)
    kn = 1e5
    checked = touching = 0
    for trial in range(150):
        a, b = rng.choice(12, 2, replace=False)
        qa, qb = synth.random_quaternions(rng, 2)
        ca = np.array([10.0, 10.0, 10.0])
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        ra = synth._bounding_radius(shapes[a])
        rb = synth._bounding_radius(shapes[b])
        cb = ca + d * rng.uniform(0.3, 1.0) * (ra + rb)
        va, fa = _world(shapes[a], qa, ca)
        vb, fb = _world(shapes[b], qb, cb)
        pen = _penetration(va, fa, vb, fb)
        if abs(pen) < 1e-6:
            continue
        o, _ = scene([ca, cb], [ra, rb], [shapes[a], shapes[b]], [0, 1], [qa, qb],
                     gravity=(0.0, 0.0, 0.0), kn=kn)
        o.step(1)
        f, _ = o.forces()
        o.close()
        depth = np.linalg.norm(f[0]) / kn
        checked += 1
        if pen < 0:
            assert depth == 0.0, (trial, pen, depth)
        else:
            touching += 1
            assert pen * (1 - 1e-9) <= depth <= pen / 0.9 * (1 + 1e-9), (trial, pen, depth)
    print("hull pairs: %d checked, %d in contact" % (checked, touching))
    assert checked > 100 and touching > 20


def _closest_on_triangle(p, a, b, c):
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = ab @ ap, ac @ ap
    if d1 <= 0 and d2 <= 0:
        return a
    bp = p - b
    d3, d4 = ab @ bp, ac @ bp
    if d3 >= 0 and d4 <= d3:
        return b
    vc = d1 * d4 - d3 * d2
    if vc <= 0 and d1 >= 0 and d3 <= 0:
        return a + ab * (d1 / (d1 - d3))
    cp = p - c
    d5, d6 = ab @ cp, ac @ cp
    if d6 >= 0 and d5 <= d6:
        return c
    vb = d5 * d2 - d1 * d6
    if vb <= 0 and d2 >= 0 and d6 <= 0:
        return a + ac * (d2 / (d2 - d6))
    va = d3 * d6 - d5 * d4
    if va <= 0 and (d4 - d3) >= 0 and (d5 - d6) >= 0:
        return b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)))
    den = 1.0 / (va + vb + vc)
    return a + ab * (vb * den) + ac * (vc * den)


def test_sphere_hull_against_closest_point():
    """A ball at random places around a rock: the restatement's overlap
    (|F| / kn from rest) is r minus the distance to the hull's nearest
    point over all its faces, or r plus the depth when the centre is
    inside."""
    rng = np.random.default_rng(12)
    shapes = synth.rock_shapes(6, seed=12)
    kn = 1e5
    checked = touching = 0
    for trial in range(150):
        k = int(rng.integers(6))
        q = synth.random_quaternions(rng, 1)[0]
        cp = np.array([10.0, 10.0, 10.0])
        rb = synth._bounding_radius(shapes[k])
        r = float(np.float32(rng.uniform(0.3, 0.6)))
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        cs = cp + d * rng.uniform(0.0, 1.0) * (rb + r)
        v, f = _world(shapes[k], q, cp)
        n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        sd = np.einsum("ij,ij->i", n, cs - v[f[:, 0]])
        if sd.max() <= 0:
            want = r - sd.max()
        else:
            dist = min(np.linalg.norm(cs - _closest_on_triangle(cs, *v[t])) for t in f)
            want = r - dist
        if abs(want) < 1e-6:
            continue
        o, _ = scene([cp, cs], [rb, r], [shapes[k]], [0, -1], [q, [1, 0, 0, 0]],
                     gravity=(0.0, 0.0, 0.0), kn=kn)
        o.step(1)
        fo, _ = o.forces()
        st = o.state()
        o.close()
        i = int(np.nonzero(st["pid"] == 1)[0][0])
        got = np.linalg.norm(fo[i]) / kn
        checked += 1
        if want < 0:
            assert got == 0.0, (trial, want, got)
        else:
            touching += 1
            assert abs(got - want) <= 1e-9 * max(1.0, want) + 1e-12, (trial, want, got)
    print("sphere-hull: %d checked, %d in contact" % (checked, touching))
    assert checked > 100 and touching > 40


def test_rock_on_triangles_counts_one_plane_once():
    """A rock pressed into a floor made of triangles: the overlap is the
    deepest vertex below the floor, along the floor's normal; a floor of two
    coplanar triangles whose shared diagonal runs under the rock gives the
    same force as one large triangle (coplanar contacts count once)."""
    rng = np.random.default_rng(13)
    shapes = synth.rock_shapes(6, seed=13)
    kn = 1e5
    z0 = 5.0
    one = [((0.0, 0.0, z0), (40.0, 0.0, z0), (0.0, 40.0, z0))]
    two = [((0.0, 0.0, z0), (20.0, 0.0, z0), (20.0, 20.0, z0)),
           ((0.0, 0.0, z0), (20.0, 20.0, z0), (0.0, 20.0, z0))]
    checked = 0
    for trial in range(40):
        k = int(rng.integers(6))
        q = synth.random_quaternions(rng, 1)[0]
        rb = synth._bounding_radius(shapes[k])
        c = np.array([10.0, 10.0, 0.0])
        v, _ = _world(shapes[k], q, np.zeros(3))
        c[2] = z0 - v[:, 2].min() - rng.uniform(1e-4, 5e-3)   # deepest vertex below the floor
        want = z0 - (c[2] + v[:, 2].min())
        forces = []
        for tris in (one, two):
            s = synth.box_system(1, 20.0, 20.0, 2.0 * rb + 0.05, 0, density=7.8e-3, kn=kn,
                                 gravity=(0.0, 0.0, 0.0))
            s.nwalls, s.tri0, s.ntris = 0, 0, len(tris)
            o = EnsRestated([s], [E.triangle(*t) for t in tris], E.LAW_LINEAR, 1e-5, 0.04, 32,
                            precision="f64")
            o.set_state(c[None, :], np.array([rb]))
            o.set_polyhedra([shapes[k]], np.array([0], np.int32), np.asarray(q)[None, :])
            o.step(1)
            f, _ = o.forces()
            o.close()
            forces.append(f[0])
        np.testing.assert_allclose(forces[0], [0.0, 0.0, kn * want], rtol=1e-9, atol=1e-12)
        np.testing.assert_array_equal(forces[0], forces[1])
        checked += 1
    assert checked == 40
