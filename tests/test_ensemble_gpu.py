"""GPU parity of the ensemble path: the sm_100a kernels through the C ABI
(include/blaze_ens.h) against the FP32 restatement (oracle/ens_oracle.c),
which follows the same operation order: states, per-particle contact forces
and torques, memory order and re-sort count are compared bit for bit."""
import numpy as np
import pytest

from bindings import EnsRestated
from blaze import ensemble as E
from blaze import synth

pytestmark = pytest.mark.gpu

DT = 1e-5
SKIN = 0.02


def compare(gpu, ora, what):
    a = gpu.state()
    b = ora.state()
    assert a["status"] == b["status"], (what, a["status"], b["status"])
    for key in ("pos", "vel", "avel", "radius"):
        np.testing.assert_array_equal(a[key].astype(np.float64), b[key], err_msg="%s %s" % (what, key))
    np.testing.assert_array_equal(a["pid"], b["pid"], err_msg=what)
    np.testing.assert_array_equal(a["sys"], b["sys"], err_msg=what)
    fa, ta = gpu.forces()
    fb, tb = ora.forces()
    np.testing.assert_array_equal(fa.astype(np.float64), fb, err_msg="%s force" % what)
    np.testing.assert_array_equal(ta.astype(np.float64), tb, err_msg="%s torque" % what)
    assert gpu.num_rebuilds() == ora.num_rebuilds(), what


def run_pair(systems, walls, pos, rad, law, checkpoints, vel=None, avel=None, use_graph=0):
    gpu = E.Ensemble(systems, walls, law=law, dt=DT, skin=SKIN, max_nbr=32, use_graph=use_graph,
                     capture_forces=1)
    ora = EnsRestated(systems, walls, law, DT, SKIN, 32, precision="f32")
    gpu.set_state(pos, rad, vel, avel)
    ora.set_state(pos, rad, vel, avel)
    done = 0
    for k in checkpoints:
        gpu.step(k - done)
        ora.step(k - done)
        done = k
        compare(gpu, ora, "step %d" % k)
    gpu.close()


@pytest.fixture(scope="module")
def boxes():
    return synth.box_ensemble([700, 1500, 300], seed=5, mus=[0.2, 0.5, 0.8],
                              restitutions=[0.3, 0.6, 0.9], height_factor=4.0)


def test_linear_history_law_bit_exact(boxes):
    S, W, p, r = boxes
    run_pair(S, W, p, r, E.LAW_LINEAR, (1, 2, 10, 150, 600))


def test_hertz_mindlin_rolling_bit_exact(boxes):
    S, W, p, r = boxes
    S = [E.System.from_buffer_copy(bytes(s)) for s in S]
    for s in S:
        s.youngs = 1e5      # 1e7 Pa
        s.poisson = 0.3
        s.mu_roll = 0.01
    rng = np.random.default_rng(11)
    avel = rng.normal(scale=50.0, size=p.shape).astype(np.float32)
    run_pair(S, W, p, r, E.LAW_HERTZ_MINDLIN, (1, 10, 400), avel=avel)


def mesh_silo(n=1500, seed=2):
    """A small silo: cylinder r = 3 cm (axis z) over a conical hopper of 64
    triangles down to a 1.2 cm outlet, a plane below, spheres r in
    [0.1, 0.2] cm on a lattice above the hopper, thrown down and sideways."""
    R, r_out, h_hop = 3.0, 0.6, 3.0
    walls = [E.cylinder((0, 0, 0), (0, 0, 1), R), E.plane((0, 0, 1), -0.5)]
    tris = []
    nseg = 32
    for k in range(nseg):
        a0, a1 = 2 * np.pi * k / nseg, 2 * np.pi * (k + 1) / nseg
        t0 = (R * np.cos(a0), R * np.sin(a0), h_hop)
        t1 = (R * np.cos(a1), R * np.sin(a1), h_hop)
        b0 = (r_out * np.cos(a0), r_out * np.sin(a0), 0.0)
        b1 = (r_out * np.cos(a1), r_out * np.sin(a1), 0.0)
        tris += [E.triangle(t0, b0, b1), E.triangle(t0, b1, t1)]
    walls += tris
    s = E.System()
    s.n = n
    cell = 0.42
    for k, (o, ext) in enumerate(zip((-R - cell, -R - cell, -1.0), (2 * R + 2 * cell,) * 2 + (14.0,))):
        s.origin[k] = o
        s.ncells[k] = int(np.ceil(ext / cell))
    s.cell = cell
    s.gravity[2] = -981.0
    s.density = 2600e-6
    s.kn, s.kt_ratio, s.youngs, s.poisson = 1e5, 2.0 / 7.0, 1e5, 0.3
    s.restitution, s.mu, s.mu_wall, s.mu_roll = 0.6, 0.5, 0.5, 0.01
    s.wall0, s.nwalls, s.tri0, s.ntris = 0, 2, 2, len(tris)
    rng = np.random.default_rng(seed)
    pts = synth.lattice_fill(4 * n, (-R + 0.25, -R + 0.25, 1.0), (R - 0.25, R - 0.25, 12.5), 0.41,
                             rng, jitter=0.01)
    pts = pts[np.hypot(pts[:, 0], pts[:, 1]) < R - 0.25]
    cone_z = (np.hypot(pts[:, 0], pts[:, 1]) - r_out) / (R - r_out) * h_hop
    pts = pts[pts[:, 2] > cone_z + 0.3][:n]
    assert len(pts) == n
    rad = rng.uniform(0.1, 0.2, n)
    vel = np.concatenate([rng.normal(scale=40.0, size=(n, 2)), np.full((n, 1), -80.0)], 1)
    return [s], walls, pts.astype(np.float32), rad.astype(np.float32), vel.astype(np.float32)


@pytest.mark.parametrize("law", [E.LAW_LINEAR, E.LAW_HERTZ_MINDLIN])
def test_triangle_mesh_and_cylinder_bit_exact(law):
    S, W, p, r, v = mesh_silo()
    run_pair(S, W, p, r, law, (1, 50, 800), vel=v)


def test_graph_stepping_equals_plain(boxes):
    S, W, p, r = boxes
    out = []
    for g in (0, 1):
        e = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=DT, skin=SKIN, use_graph=g)
        e.set_state(p, r)
        e.step(403)
        out.append(e.state())
        e.close()
    for key in ("pos", "vel", "avel", "pid"):
        np.testing.assert_array_equal(out[0][key], out[1][key])
    assert out[0]["status"] == 0 and out[1]["status"] == 0


def turning_drum(n=1500, seed=3):
    """A small ball mill as a turning triangle mesh: drum R = 8 cm, L = 4 cm
    (48 x 4 barrel quads and 4 lifters 1.5 x 1.2 cm: 480 triangles; the end
    plates are planes turning in place) turning at 60 rpm about z, spheres
    r in [0.15, 0.3] cm packed against the lower barrel, thrown down at
    50 cm/s; y vertical."""
    R, L = 8.0, 4.0
    tris = synth.drum_mesh_triangles(R, L, 48, 4, n_lifters=4, lifter_w=1.5, lifter_h=1.2,
                                     end_fans=False)
    walls = [E.plane((0, 0, 1), 0.0), E.plane((0, 0, -1), -L)] + [E.triangle(*t) for t in tris]
    s = E.System()
    s.n = n
    cell = 0.64
    for k, (o, ext) in enumerate(zip((-R - cell, -R - cell, -cell),
                                     (2 * R + 2 * cell, 2 * R + 2 * cell, L + 2 * cell))):
        s.origin[k] = o
        s.ncells[k] = int(np.ceil(ext / cell))
    s.cell = cell
    s.gravity[1] = -981.0
    s.density = 7800e-6
    s.kn, s.kt_ratio, s.youngs, s.poisson = 1e5, 2.0 / 7.0, 1e6, 0.3
    s.restitution, s.mu, s.mu_wall, s.mu_roll = 0.4, 0.6, 0.6, 0.01
    s.wall0, s.nwalls, s.tri0, s.ntris = 0, 2, 2, len(tris)
    s.rot_axis[2] = 1.0
    s.rot_omega = 2.0 * np.pi
    rng = np.random.default_rng(seed)
    pts = synth.lattice_fill(2400, (-R + 0.35, -R + 0.35, 0.35), (R - 0.35, 0.0, L - 0.35), 0.62,
                             rng, jitter=0.01)
    pts = pts[np.hypot(pts[:, 0], pts[:, 1]) < R - 0.35]
    pts = pts[np.argsort(pts[:, 1], kind="stable")][:n]
    assert len(pts) == n
    rad = rng.uniform(0.15, 0.3, n)
    vel = np.zeros((n, 3))
    vel[:, 1] = -50.0
    return [s], walls, pts.astype(np.float32), rad.astype(np.float32), vel.astype(np.float32)


@pytest.mark.parametrize("law", [E.LAW_LINEAR, E.LAW_HERTZ_MINDLIN])
def test_turning_drum_mesh_bit_exact(law):
    """Triangles turning with the drum (tested in its frame, surfaces moving):
    GPU = FP32 restatement bit for bit, graph stepping included; and the
    turn is felt (the mean tangential velocity of the charge follows the
    drum)."""
    S, W, p, r, v = turning_drum()
    run_pair(S, W, p, r, law, (1, 50, 400), vel=v)
    run_pair(S, W, p, r, law, (8, 64), vel=v, use_graph=1)
    e = E.Ensemble(S, W, law=law, dt=DT, skin=SKIN, use_graph=1)
    e.set_state(p, r, v)
    e.step(2000)
    st = e.state()
    e.close()
    assert st["status"] == 0, st["status"]
    x, y = st["pos"][:, 0].astype(np.float64), st["pos"][:, 1].astype(np.float64)
    vt = (x * st["vel"][:, 1] - y * st["vel"][:, 0]) / np.hypot(x, y)   # counter-clockwise
    assert vt.mean() > 1.0, vt.mean()


@pytest.mark.parametrize("law", [E.LAW_LINEAR, E.LAW_HERTZ_MINDLIN])
def test_persistent_stepping_equals_plain(boxes, law):
    """use_graph = 2: one persistent kernel runs the steps between re-sorts
    with a grid barrier per step.  Same states, order and re-sort count as
    plain stepping, over uneven calls (budgets that end on and off a
    re-sort); planes, and the triangle-mesh silo with its cylinder."""
    S, W, p, r = boxes
    # velocities that make the boxes re-sort every few tens of steps
    v = np.random.default_rng(9).normal(scale=10.0, size=p.shape).astype(np.float32)
    S2, W2, p2, r2, v2 = mesh_silo()
    for (sy, wa, pos, rad, vel) in ((S, W, p, r, v), (S2, W2, p2, r2, v2)):
        out, rb = [], []
        for g in (0, 2):
            e = E.Ensemble(sy, wa, law=law, dt=DT, skin=SKIN, use_graph=g)
            e.set_state(pos, rad, vel)
            for k in (1, 7, 150, 245):
                e.step(k)
            out.append(e.state())
            rb.append(e.num_rebuilds())
            e.close()
        for key in ("pos", "vel", "avel", "pid"):
            np.testing.assert_array_equal(out[0][key], out[1][key], err_msg=key)
        assert out[0]["status"] == 0 and out[1]["status"] == 0, (out[0]["status"], out[1]["status"])
        assert rb[0] == rb[1] and rb[0] > 1, rb


def test_out_of_grid_is_reported_not_faulted(boxes):
    S, W, p, r = boxes
    p = p.copy()
    p[3] = (500.0, 500.0, 500.0)
    e = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=DT, skin=SKIN, use_graph=0)
    e.set_state(p, r)
    e.step(2)
    assert e.sync() & 2
    e.close()


def test_barrier_wait_gives_up_and_the_context_stays_usable(boxes):
    """Persistent stepping's grid barrier waits at most 2 s: two blocks at a
    barrier counted for three (nothing completes it) give up, raise status
    16 and return; the next ensemble runs normally on the same context."""
    lib = E.load()
    lib.blaze_ens_check_barrier_timeout.argtypes = []
    assert lib.blaze_ens_check_barrier_timeout() == 16
    S, W, p, r = boxes
    e = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=DT, skin=SKIN, use_graph=2)
    e.set_state(p, r)
    e.step(20)
    assert e.sync() == 0
    e.close()
