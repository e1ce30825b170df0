"""GPU parity through the C ABI: the sm_100a kernels against the reference's
own kernels (golden fixtures) and against the FP32 restatement, bit for bit
in the reference mode (skin 0); within stated tolerance with a Verlet skin."""
import ctypes

import numpy as np
import pytest

from bindings import Restated
from blaze import device, synth

pytestmark = pytest.mark.gpu

FORCE_KEYS = ("f_pp", "t_pp", "f_wall", "t_wall", "f_lift", "t_lift")


def gpu_sim(g, **opts):
    s = device.Simulation(sim_info=g.sim_info, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                          dobj=g.dobj, n_d=g.n_d, **opts)
    s.set_cylinder_rotation(g.cyl_rot)
    st = g.init()
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    return s


def test_golden_bit_exact(golden):
    s = gpu_sim(golden, capture_forces=1)
    done = 0
    for k in golden.checkpoints:
        s.step(k - done)
        done = k
        ref = golden.at(k)
        st = s.state()
        assert st["status"] == 0, device.decode_status(st["status"])
        for key in ("pos", "vel", "avel"):
            np.testing.assert_array_equal(st[key], ref[key], err_msg="%s step %d" % (key, k))
        np.testing.assert_array_equal(st["pid"], ref["pid"])
        np.testing.assert_array_equal(st["type"], ref["type"])
        f = s.forces()
        for key in FORCE_KEYS:
            np.testing.assert_array_equal(f[key], ref[key], err_msg="%s step %d" % (key, k))
        nn, lst = s.nlist()
        np.testing.assert_array_equal(nn, ref["nn"], err_msg="contact counts step %d" % k)
        w = ref["list"].shape[1]
        np.testing.assert_array_equal(lst[:, :w], ref["list"], err_msg="contact lists step %d" % k)
    s.close()


@pytest.fixture(scope="module")
def box(tmp_path_factory):
    return synth.box_project(str(tmp_path_factory.mktemp("box")))


def test_box_bit_exact_vs_restatement(box):
    P, st0 = box
    s = device.Simulation(P, capture_forces=1)
    s.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
    o = Restated("f32").init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d)
    o.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
    for chunk in (1, 9, 40):
        s.step(chunk)
        assert o.step(chunk) == 0
        a, b = s.state(), o.state()
        assert a["status"] == 0
        for key in ("pos", "vel", "avel"):
            np.testing.assert_array_equal(a[key].astype(np.float64), b[key])
        np.testing.assert_array_equal(a["pid"], b["pid"])
        fa, fb = s.forces(), o.forces()
        for key in FORCE_KEYS:
            np.testing.assert_array_equal(fa[key].astype(np.float64), fb[key])
    s.close()


def test_box_reference_abi_kdevice(box):
    """The reference-facing entry points (Part 1) drive the same step."""
    P, st0 = box
    kd = device.KDevice(P.wobj, P.pobj, P.dobj, P.n_w, P.n_p, P.n_d, P.sim_info, P.init)
    pos = np.ascontiguousarray(st0["pos"], np.float32)
    vel = np.ascontiguousarray(st0["vel"], np.float32)
    avel = np.ascontiguousarray(st0["avel"], np.float32)
    kd.IDevice_Set_ParticleSystem_State(pos, None, vel, avel, None, st0["type"], st0["pid"])
    for _ in range(20):
        kd.IDevice_DEM_UpdateSim()
    n = P.num_particles
    out = {k: np.zeros((n, 3), np.float32) for k in ("pos", "vel", "avel", "acc")}
    typ = np.zeros(n, np.uint32)
    pid = np.zeros(n, np.int32)
    rc = kd.IDevice_Get_System_State(out["pos"], None, out["vel"], out["avel"], out["acc"], typ, pid)
    assert rc == 0
    o = Restated("f32").init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d)
    o.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
    o.step(20)
    b = o.state()
    np.testing.assert_array_equal(out["pos"].astype(np.float64), b["pos"])
    np.testing.assert_array_equal(pid, b["pid"])
    kd.clean()


def test_skin_mode_matches_reference_mode(box):
    """With a Verlet skin the contact set is the same; summation order only
    changes once particles change cells between rebuilds."""
    P, st0 = box
    ref = device.Simulation(P, capture_forces=1)
    fast = device.Simulation(P, capture_forces=1, skin=0.02)
    for s in (ref, fast):
        s.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
    ref.step(1)
    fast.step(1)
    for key in FORCE_KEYS:
        np.testing.assert_array_equal(ref.forces()[key], fast.forces()[key])
    ref.step(199)
    fast.step(199)
    a, b = ref.state(), fast.state()
    assert a["status"] == 0 and b["status"] == 0
    ia, ib = np.argsort(a["pid"]), np.argsort(b["pid"])
    scale = np.abs(a["vel"]).max()
    np.testing.assert_allclose(b["vel"][ib], a["vel"][ia], rtol=0, atol=1e-4 * scale)
    np.testing.assert_allclose(b["pos"][ib], a["pos"][ia], rtol=0, atol=1e-5)
    assert fast.num_rebuilds() < ref.num_rebuilds()
    ref.close()
    fast.close()


def _skin_vs_reference_each_step(P, st, skin, pre, count, hatch=False):
    """Step the skin path `pre` steps, then for `count` steps compare each
    step's particle-particle forces with the reference mode's from the same
    state: equal up to the order of summation (a pair the list missed
    would show as a whole contact force)."""
    sk = device.Simulation(P, skin=skin, capture_forces=1)
    rf = device.Simulation(P, capture_forces=1)
    for s in (sk, rf):
        if hatch:
            s.open_hatch()
    sk.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    sk.step(pre)
    mass = np.array([P.pobj[t].mass for t in range(P.n_p)], np.float64)
    worst = 0.0
    for _ in range(count):
        a = sk.state()
        rf.set_state(a["pos"], a["vel"], a["avel"], a["type"], a["pid"])
        rf.step(1)
        fr, pr = rf.forces()["f_pp"], rf.state()["pid"]
        sk.step(1)
        fs, ps = sk.forces()["f_pp"], sk.state()["pid"]
        x = fr[np.argsort(pr)].astype(np.float64)
        y = fs[np.argsort(ps)].astype(np.float64)
        w = mass[a["type"][np.argsort(a["pid"])]] * 981.0
        e = np.linalg.norm(x - y, axis=1) / np.maximum(np.linalg.norm(x, axis=1), w)
        worst = max(worst, float(e.max()))
    status = sk.sync()
    sk.close()
    rf.close()
    return worst, status


def test_skin_list_finds_every_contact_box(box):
    """The box (r = 0.1 cm, project cells 0.2 cm = 2 r) with a 0.02 cm skin,
    in its bouncing phase (steps 6,000-6,200): the list grid's cells are
    2 r + skin, so no pair within the skin lies beyond the 27 cells."""
    P, st0 = box
    worst, status = _skin_vs_reference_each_step(P, st0, 0.02, 6000, 200)
    assert status == 0, device.decode_status(status)
    assert worst < 1e-4, worst


def test_skin_list_finds_every_contact_silo(silo_small):
    """The silo workload (r in [0.2, 0.4] cm, project cells 0.8 cm = 2 r_max)
    with the headline's 0.16 cm skin, hatch open, steps 3,000-3,100."""
    P, st = silo_small
    worst, status = _skin_vs_reference_each_step(P, st, 0.16, 3000, 100, hatch=True)
    assert status == 0, device.decode_status(status)
    assert worst < 1e-4, worst


def test_status_out_of_grid_and_overflow(box):
    P, st0 = box
    pos = st0["pos"].copy()
    pos[5] = (50.0, 50.0, 50.0)  # outside the hash grid
    s = device.Simulation(P, max_nbr=2, skin=0.5)
    s.set_state(pos, st0["vel"], st0["avel"], st0["type"], st0["pid"])
    s.step(1)
    st = s.sync()
    assert st & 2, device.decode_status(st)   # out of grid, reported, no fault
    assert st & 1, device.decode_status(st)   # neighbour overflow, reported
    s.close()


@pytest.fixture(scope="module")
def silo_small(tmp_path_factory):
    return synth.silo_project(str(tmp_path_factory.mktemp("silo")), n=20000)


def run_steps(P, st, steps, **opts):
    s = device.Simulation(P, **opts)
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    s.open_hatch()
    s.step(steps)
    out = s.state()
    s.close()
    return out


def test_wall_culling_is_exact(silo_small):
    """Per-cell wall-op lists drop only ops that cannot touch the cell."""
    P, st = silo_small
    a = run_steps(P, st, 300, wall_grid=0)
    b = run_steps(P, st, 300, wall_grid=1)
    assert a["status"] == 0 and b["status"] == 0
    for key in ("pos", "vel", "avel", "pid"):
        np.testing.assert_array_equal(a[key], b[key])


@pytest.mark.parametrize("skin", [0.0, 0.04])
def test_graph_stepping_is_exact(silo_small, skin):
    """The CUDA-graph path (IF node around the re-sort) equals plain stepping."""
    P, st = silo_small
    a = run_steps(P, st, 301, skin=skin, use_graph=0)
    b = run_steps(P, st, 301, skin=skin, use_graph=1)
    for key in ("pos", "vel", "avel", "pid"):
        np.testing.assert_array_equal(a[key], b[key])


def test_graph_stepping_uneven_calls(silo_small):
    """Graph stepping with a skin cut into calls of uneven length (tails
    shorter than a block run as one-step graphs, blocks start mid-call)
    equals plain stepping bit for bit, and neither runs an exact block on
    this slow state."""
    P, st = silo_small
    a = run_steps(P, st, 203, skin=0.04, use_graph=0)
    s = device.Simulation(P, skin=0.04, use_graph=1)
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    s.open_hatch()
    s.prepare_graphs()
    for k in (5, 3, 13, 1, 8, 20, 7, 9, 16, 2, 40, 79):
        s.step(k)
    b = s.state()
    assert s.num_exact_blocks() == 0
    s.close()
    assert a["status"] == 0 and b["status"] == 0
    for key in ("pos", "vel", "avel", "pid"):
        np.testing.assert_array_equal(a[key], b[key])


def test_graph_stepping_exact_blocks_fast_state(box):
    """A state too fast for an 8-step block without list checks (speeds
    N(0, 300 cm/s) against a 0.02 cm skin at dt 1e-5 s): the blocks run
    exact, with a check before every step.  Graph and plain stepping re-sort
    at the same steps and agree bit for bit, and no stale-list status is
    raised."""
    P, st0 = box
    vel = np.random.default_rng(7).normal(scale=300.0, size=st0["vel"].shape).astype(np.float32)
    out = []
    for g in (0, 1):
        s = device.Simulation(P, skin=0.02, use_graph=g)
        s.set_state(st0["pos"], vel, st0["avel"], st0["type"], st0["pid"])
        s.step(67)
        out.append((s.state(), s.num_rebuilds(), s.num_exact_blocks()))
        s.close()
    (a, ra, xa), (b, rb, xb) = out
    assert a["status"] == 0 and b["status"] == 0, device.decode_status(a["status"] | b["status"])
    # steps 0-7 check after every step (forced re-sort at set_state); the
    # block starts 8, 16, ..., 64 all run exact, in both stepping modes
    assert xa == xb == 8, (xa, xb)
    assert ra == rb and ra > 67 // 8
    for key in ("pos", "vel", "avel", "pid"):
        np.testing.assert_array_equal(a[key], b[key])


@pytest.mark.gpu
def test_shared_reciprocal_division_is_ieee():
    """div3_rn (one correctly rounded reciprocal + two corrections per
    quotient, dem_common.cuh) equals IEEE division bit for bit on 3 x 2^30
    random quotients over 1e-25..1e25 / 1e-18..1e18 (including the ranges
    it hands to the IEEE division), zero and power-of-two numerators."""
    lib = device.load()
    lib.blaze_check_division.restype = ctypes.c_longlong
    lib.blaze_check_division.argtypes = [ctypes.c_longlong, ctypes.c_ulonglong]
    assert lib.blaze_check_division(1 << 30, 12345) == 0


def test_moving_walls_enter_the_list_check(tmp_path):
    """A drum turning at 30 rpm (wall and lifter surface speed up to 157
    cm/s) with a 0.015 cm skin at dt 2e-6 s: from the first block start the
    list check counts that surface speed as a particle speed, so every block
    runs exact although the charge starts at rest (a lifter can set a resting
    sphere in motion within a block).  Graph and plain stepping agree bit for
    bit, and no stale-list status is raised."""
    P, st = synth.mill_project(str(tmp_path), n=3000)
    R = float(P.wobj[0].cyl_geo.radius)
    rad = float(P.mill.RadPerStep)
    out = []
    for g in (0, 1):
        s = device.Simulation(P, skin=0.015, use_graph=g)
        s.set_cylinder_rotation(True)
        s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
        s.set_dobj_rotation(R, R, rad)
        s.step(64)
        out.append((s.state(), s.num_exact_blocks()))
        s.close()
    (a, xa), (b, xb) = out
    assert a["status"] == 0 and b["status"] == 0, device.decode_status(a["status"] | b["status"])
    assert xa == xb == 7, (xa, xb)   # block starts 8, 16, ..., 56
    for key in ("pos", "vel", "avel", "pid"):
        np.testing.assert_array_equal(a[key], b[key])


@pytest.mark.parametrize("use_graph", [0, 1])
def test_stale_list_status_raised(box, use_graph):
    """A box of resting spheres keeps its list through a block (no check
    inside it); then the whole box is moved 0.21 cm up between two calls,
    into the bottom layer.  The spheres it strikes leave at thousands of cm/s
    within the block, past half the 0.02 cm skin before the next check, and
    the step reports it as status bit 64 (stale list) instead of silently
    missing contacts."""
    P, st0 = box
    s = device.Simulation(P, skin=0.02, use_graph=use_graph)
    s.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
    s.step(16)
    assert s.sync() == 0
    w = s.wobj()
    for k in range(w[0].num_vertex):
        w[0].vertex[k].z += 0.21
    for f in range(w[0].num_surfaces):
        w[0].surfaces[f].centroid.z += 0.21
    s.update_wobj(w, P.n_w)
    s.step(8)
    st = s.sync()
    s.close()
    assert st & 64, device.decode_status(st)
