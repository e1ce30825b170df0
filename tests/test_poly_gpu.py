"""Convex polyhedra on the GPU through the C ABI, against the reference's own
polyhedron kernels: the oracle-A fixtures (tests/golden/box_poly.npz, 1,440
dodecahedra of the reference's Poly_1cm object in its Container_128 box;
drum_poly.npz, 1,200 in the rotating 90 cm mill drum with end plates;
lifter_poly.npz, the same drum with its eight Square_Lifter16 volume
objects), random orientations and spins, contacts of every kind from the
first step; and variants run against oracle A live (oracle/_ref travels with
the repository): rotation off, 2-D mode, an infinite plane after a face.

Bar: bit for bit at every checkpoint (contact lists, particle-particle and
wall forces and torques, positions, velocities, spins, orientations).  The
orientation update's half-angle sine and cosine are evaluated differently
from the reference's (csrc/poly_kernels.cu, quat_step); on this fixture they
agree with the host library's everywhere."""
import ctypes

import numpy as np
import pytest

import bindings
from blaze import device
from blaze import types as T
from conftest import Golden

pytestmark = pytest.mark.gpu

STATE_KEYS = ("pos", "quat", "vel", "avel")
FORCE_KEYS = ("f_pp", "t_pp", "f_wall", "t_wall", "f_lift", "t_lift")


def gpu_sim(g, **opts):
    s = device.Simulation(sim_info=g.sim_info, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                          dobj=g.dobj, n_d=g.n_d, **opts)
    s.set_cylinder_rotation(g.cyl_rot)
    st = g.init()
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"], quat=st["quat"])
    return s


def mismatches(a, b):
    return int(np.count_nonzero(np.asarray(a) != np.asarray(b)))


def test_poly_first_step_bit_exact(golden_poly):
    g = golden_poly
    s = gpu_sim(g, capture_forces=1)
    s.step(1)
    ref = g.at(1)
    st = s.state()
    assert st["status"] == 0, device.decode_status(st["status"])
    np.testing.assert_array_equal(st["pid"], ref["pid"])
    np.testing.assert_array_equal(st["type"], ref["type"])
    nn, lst = s.nlist()
    np.testing.assert_array_equal(nn, ref["nn"])
    w = ref["list"].shape[1]
    np.testing.assert_array_equal(lst[:, :w], ref["list"])
    f = s.forces()
    for key in FORCE_KEYS:
        np.testing.assert_array_equal(f[key], ref[key], err_msg=key)
    for key in STATE_KEYS:
        np.testing.assert_array_equal(st[key], ref[key], err_msg=key)
    s.close()


def test_poly_checkpoints_bit_exact(golden_poly):
    g = golden_poly
    s = gpu_sim(g, capture_forces=1)
    done = 0
    for k in g.checkpoints:
        s.step(k - done)
        done = k
        ref = g.at(k)
        st = s.state()
        assert st["status"] == 0, device.decode_status(st["status"])
        # same memory order as the reference (the re-sort is the same stable sort)
        np.testing.assert_array_equal(st["pid"], ref["pid"], err_msg="pid %d" % k)
        nn, _ = s.nlist()
        np.testing.assert_array_equal(nn, ref["nn"], err_msg="contact counts %d" % k)
        f = s.forces()
        for key in STATE_KEYS:
            assert mismatches(st[key], ref[key]) == 0, "%s step %d" % (key, k)
        for key in FORCE_KEYS:
            assert mismatches(f[key], ref[key]) == 0, "%s step %d" % (key, k)
    s.close()


def test_poly_graph_and_skin_modes(golden_poly):
    """CUDA-graph stepping reproduces plain stepping bit for bit; a Verlet
    skin on the bounding spheres (searched on cells of 2 r + skin, so the
    contacts are summed in another order) keeps the first step's forces
    within 1e-6 of the largest and the trajectory within 1e-5 of the
    reference mode after 10 steps, 1e-3 after 50."""
    g = golden_poly
    plain = gpu_sim(g)
    graph = gpu_sim(g, use_graph=1)
    plain.step(24)
    graph.step(24)
    a, b = plain.state(), graph.state()
    for key in STATE_KEYS + ("pid",):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    ref = gpu_sim(g, capture_forces=1)
    skin = gpu_sim(g, capture_forces=1, skin=0.05)
    ref.step(1)
    skin.step(1)
    fr, fs = ref.forces(), skin.forces()
    ir, is_ = np.argsort(ref.state()["pid"]), np.argsort(skin.state()["pid"])
    for key in FORCE_KEYS:
        x, y = fr[key][ir].astype(np.float64), fs[key][is_].astype(np.float64)
        scale = max(float(np.abs(x).max()), 1e-30)
        np.testing.assert_allclose(y, x, rtol=0, atol=1e-6 * scale, err_msg=key)
    ref_done = [1]
    # the summation orders differ, and a polyhedron contact's feature can
    # flip on a rounding difference: 1e-5 of the largest value after 10
    # steps, 1e-3 after 50
    for steps, tol in ((10, 1e-5), (50, 1e-3)):
        ref.step(steps - ref_done[0])
        skin.step(steps - ref_done[0])
        ref_done[0] = steps
        a, b = ref.state(), skin.state()
        assert a["status"] == 0 and b["status"] == 0
        ia, ib = np.argsort(a["pid"]), np.argsort(b["pid"])
        for key in STATE_KEYS:
            scale = max(float(np.abs(a[key]).max()), 1e-30)
            np.testing.assert_allclose(b[key][ib], a[key][ia], rtol=0, atol=tol * scale,
                                       err_msg="%s after %d steps" % (key, steps))
    assert skin.num_rebuilds() < ref.num_rebuilds()
    for s in (plain, graph, ref, skin):
        s.close()


def test_poly_reference_abi(golden_poly):
    """Part 1 (Device_Set_System_State with orientations, Device_DEM_UpdateSim,
    Device_Get_System_State) drives the same step as the handle API."""
    g = golden_poly
    st0 = g.init()
    kd = device.KDevice(g.wobj, g.pobj, g.dobj, g.n_w, g.n_p, g.n_d, g.sim_info, None)
    kd.IDevice_drum_rotation(g.cyl_rot)
    pos = np.ascontiguousarray(st0["pos"], np.float32)
    quat = np.ascontiguousarray(st0["quat"], np.float32)
    vel = np.ascontiguousarray(st0["vel"], np.float32)
    avel = np.ascontiguousarray(st0["avel"], np.float32)
    kd.IDevice_Set_ParticleSystem_State(pos, quat, vel, avel, None, st0["type"], st0["pid"])
    for _ in range(10):
        kd.IDevice_DEM_UpdateSim()
    n = g.n
    out = {k: np.zeros((n, 3), np.float32) for k in ("pos", "vel", "avel", "acc")}
    q = np.zeros((n, 4), np.float32)
    typ = np.zeros(n, np.uint32)
    pid = np.zeros(n, np.int32)
    rc = kd.IDevice_Get_System_State(out["pos"], q, out["vel"], out["avel"], out["acc"], typ, pid)
    assert rc == 0
    kd.clean()
    s = gpu_sim(g)
    s.step(10)
    b = s.state()
    np.testing.assert_array_equal(out["pos"], b["pos"])
    np.testing.assert_array_equal(q, b["quat"])
    np.testing.assert_array_equal(pid, b["pid"])
    s.close()


need_ref_lib = pytest.mark.skipif(not bindings.ref_available(), reason="oracle/_ref not built")


def box_variant(g, kind):
    """The box fixture's structs with one setting changed."""
    si = T.SimulationInfo.from_buffer_copy(bytes(g.sim_info))
    wobj = (T.WOBJ * 8).from_buffer_copy(bytes(g.wobj))
    n_w = g.n_w
    if kind == "no_rotation":
        si.Rotation = False
    elif kind == "mode2d":
        si.Mode2D = True
    elif kind == "plane_after_face":
        # a second world object: a copy of the floor face, then an infinite
        # plane (area -1), for which the reference has no polyhedron test and
        # re-applies the contact the floor copy left behind
        W = wobj[1]
        ctypes.memmove(ctypes.addressof(W), ctypes.addressof(wobj[0]), ctypes.sizeof(T.WOBJ))
        W.num_surfaces = 2
        W.surfaces[0] = wobj[0].surfaces[0]
        W.surfaces[1] = wobj[0].surfaces[0]
        W.surfaces[1].area = -1.0
        n_w = 2
        si.Num_WorldObjects = 2
    return si, wobj, n_w


@need_ref_lib
@pytest.mark.parametrize("kind", ["no_rotation", "mode2d", "plane_after_face"])
def test_poly_variants_vs_live_reference(kind):
    g = Golden("box_poly")
    si, wobj, n_w = box_variant(g, kind)
    st0 = g.init()
    R = bindings.RefHost()
    R.init(si, wobj, n_w, g.pobj, g.n_p, g.dobj, g.n_d, threads=8, capture=True)
    R.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"], quat=st0["quat"])
    s = device.Simulation(sim_info=si, wobj=wobj, n_w=n_w, pobj=g.pobj, n_p=g.n_p, dobj=g.dobj,
                          n_d=g.n_d, capture_forces=1)
    s.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"], quat=st0["quat"])
    for chunk in (1, 9):
        assert R.step(chunk) == 0
        s.step(chunk)
        a, b = s.state(), R.state()
        assert a["status"] == 0, device.decode_status(a["status"])
        np.testing.assert_array_equal(a["pid"], b["pid"])
        for key in STATE_KEYS:
            assert mismatches(a[key], b[key]) == 0, "%s %s" % (kind, key)
        fa, fb = s.forces(), R.forces()
        for key in FORCE_KEYS:
            assert mismatches(fa[key], fb[key]) == 0, "%s %s" % (kind, key)
        if chunk == 1:  # the first step has floor contacts to compare
            assert int((np.abs(fb["f_wall"]).sum(axis=1) > 0).sum()) > 20
    s.close()


@need_ref_lib
@pytest.mark.parametrize("name", ["drum_poly", "lifter_poly"])
def test_poly_energy_tallies_vs_live_reference(name):
    """Energy tallies (EnergyCalc on) of polyhedra in the drum, with and
    without the lifters: the GPU's FP64 sums equal oracle A's FP64 sums of
    the same per-contact FP32 values (the reference's polyhedron kernel adds
    them through the same response functions) within 1e-9, and the state
    stays bit for bit."""
    g = Golden(name)
    si = T.SimulationInfo.from_buffer_copy(bytes(g.sim_info))
    si.EnergyCalc = True
    st0 = g.init()
    R = bindings.RefHost()
    R.init(si, g.wobj, g.n_w, g.pobj, g.n_p, g.dobj, g.n_d, threads=8, capture=False)
    R.set_cylinder_rotation(g.cyl_rot)
    R.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"], quat=st0["quat"])
    R.reset_energy()
    s = device.Simulation(sim_info=si, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                          dobj=g.dobj, n_d=g.n_d, use_graph=1)
    s.set_cylinder_rotation(g.cyl_rot)
    s.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"], quat=st0["quat"])
    s.reset_energy()
    for chunk in (1, 9, 40):
        assert R.step(chunk) == 0
        s.step(chunk)
        a, b = s.state(), R.state()
        for key in STATE_KEYS:
            assert mismatches(a[key], b[key]) == 0, key
        ref = R.energy64()
        assert np.all(ref[[0, 2]] > 0)
        np.testing.assert_allclose(s.energy(), ref, rtol=1e-9)
    s.close()
