"""Convex polyhedra on the GPU through the C ABI, against the reference's own
polyhedron kernels (oracle A fixture tests/golden/box_poly.npz: 1,440
dodecahedra of the reference's Poly_1cm object in its Container_128 box,
random orientations and spins, contacts of every kind from the first step).

Bar: bit for bit at every checkpoint (contact lists, particle-particle and
wall forces and torques, positions, velocities, spins, orientations).  The
orientation update's half-angle sine and cosine are evaluated differently
from the reference's (csrc/poly_kernels.cu, quat_step); on this fixture they
agree with the host library's everywhere."""
import numpy as np
import pytest

from blaze import device

pytestmark = pytest.mark.gpu

STATE_KEYS = ("pos", "quat", "vel", "avel")
FORCE_KEYS = ("f_pp", "t_pp", "f_wall", "t_wall", "f_lift", "t_lift")


def gpu_sim(g, **opts):
    s = device.Simulation(sim_info=g.sim_info, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                          dobj=g.dobj, n_d=g.n_d, **opts)
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
    skin on the bounding spheres keeps the first step's forces bit for bit
    and the trajectory within 1e-5 of the reference mode."""
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
    for key in FORCE_KEYS:
        np.testing.assert_array_equal(fr[key], fs[key], err_msg=key)
    ref.step(49)
    skin.step(49)
    a, b = ref.state(), skin.state()
    assert a["status"] == 0 and b["status"] == 0
    ia, ib = np.argsort(a["pid"]), np.argsort(b["pid"])
    for key in STATE_KEYS:
        scale = max(float(np.abs(a[key]).max()), 1e-30)
        np.testing.assert_allclose(b[key][ib], a[key][ia], rtol=0, atol=1e-5 * scale, err_msg=key)
    assert skin.num_rebuilds() < ref.num_rebuilds()
    for s in (plain, graph, ref, skin):
        s.close()


def test_poly_reference_abi(golden_poly):
    """Part 1 (Device_Set_System_State with orientations, Device_DEM_UpdateSim,
    Device_Get_System_State) drives the same step as the handle API."""
    g = golden_poly
    st0 = g.init()
    kd = device.KDevice(g.wobj, g.pobj, g.dobj, g.n_w, g.n_p, g.n_d, g.sim_info, None)
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
