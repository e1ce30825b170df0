"""One revolution of the reference's ball mill on the GPU against oracle A.

Fixture: tests/golden/mill_power.npz (tests/golden/make_mill_power.py): the
reference's `Mill_SPH30` world (242 spheres in the 90 cm drum, eight
Square_Lifter16 lifters, 22 rpm, dt 1e-5 s, energy tallies on), run by
oracle A for the 272,727 steps of the first revolution with the drum
rotating and the mill driver's lifter turn before every step.

The GPU run turns the lifters on the device (blaze_set_dobj_rotation) and
keeps the tallies in FP64.  Bar: state (positions, velocities, spins,
P_ID, memory order) and lifter vertices bit for bit at every checkpoint,
after one revolution included; tallies equal to oracle A's FP64 sums of the
same per-contact FP32 values within 1e-9 (only the summation order
differs).  The reference's own FP32 tallies and its published powers are
checked in tests/test_oracle_golden.py (the oracle's pin).
"""
import numpy as np
import pytest

from blaze import device
from conftest import Golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mill():
    return Golden("mill_power")


def test_one_revolution_bit_exact(mill):
    g = mill
    z = g.z
    s = device.Simulation(sim_info=g.sim_info, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                          dobj=g.dobj, n_d=g.n_d, use_graph=1)
    s.set_cylinder_rotation(True)
    st = g.init()
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    s.reset_energy()
    about = float(z["about"])
    s.set_dobj_rotation(about, about, float(z["rad_per_step"]))
    done = 0
    for k in [int(x) for x in z["checkpoints"]]:
        s.step(k - done)
        done = k
        a = s.state()
        assert a["status"] == 0, device.decode_status(a["status"])
        for key in ("pos", "vel", "avel", "pid"):
            np.testing.assert_array_equal(a[key], z["s%d_%s" % (k, key)],
                                          err_msg="%s after %d steps" % (key, k))
        d = s.dobj()
        vert = np.array([[[d[q].vertex[v].x, d[q].vertex[v].y, d[q].vertex[v].z]
                           for v in range(8)] for q in range(g.n_d)], np.float32)
        np.testing.assert_array_equal(vert, z["s%d_lifter_vertex" % k],
                                      err_msg="lifters after %d steps" % k)
        e = s.energy()
        ref = z["s%d_energy64" % k]
        np.testing.assert_allclose(e, ref, rtol=1e-9, err_msg="tallies after %d steps" % k)
    nspr = int(z["steps_per_rev"])
    T = nspr * float(z["dt"])
    e = s.energy()
    print("GPU power after one revolution (FP64 tallies): total %.3f particle %.3f lifter %.3f "
          "drum %.3f W" % (e.sum() / T, e[0] / T, e[1] / T, e[2] / T))
    s.close()


def test_reference_energy_interface(mill):
    """Device_Reset_Energy / Device_Get_Energy / Device_Set_Tallys through the
    reference interface: Device_Get_Energy returns the FP64 tallies rounded
    to FP32, in GetEnergy's units; the handle API's run of the same 100 steps
    has the same tallies."""
    g = mill
    st = g.init()
    kd = device.KDevice(g.wobj, g.pobj, g.dobj, g.n_w, g.n_p, g.n_d, g.sim_info, None)
    kd.IDevice_drum_rotation(True)
    pos = np.ascontiguousarray(st["pos"], np.float32)
    vel = np.ascontiguousarray(st["vel"], np.float32)
    avel = np.ascontiguousarray(st["avel"], np.float32)
    kd.IDevice_Set_ParticleSystem_State(pos, None, vel, avel, None, st["type"], st["pid"])
    kd.IDevice_Mill_reset_energy(0)
    for _ in range(100):
        kd.IDevice_DEM_UpdateSim()
    e = np.zeros(3, np.float32)
    assert kd.IDevice_Get_Energy(e) == 0
    assert np.all(e > 0)
    kd.IDevice_Set_Tallys(np.array([1e4, 2e4, 3e4], np.float32))
    e2 = np.zeros(3, np.float32)
    kd.IDevice_Get_Energy(e2)
    np.testing.assert_array_equal(e2, np.array([1.0, 2.0, 3.0], np.float32))
    kd.IDevice_Mill_reset_energy(0)
    kd.IDevice_Get_Energy(e2)
    assert np.all(e2 == 0)
    kd.clean()
    s = device.Simulation(sim_info=g.sim_info, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                          dobj=g.dobj, n_d=g.n_d)
    s.set_cylinder_rotation(True)
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    s.reset_energy()
    s.step(100)
    np.testing.assert_array_equal(s.energy().astype(np.float32), e)
    s.close()


def test_state_file_round_trip(mill, tmp_path):
    """blaze_write_state on the GPU simulation: the file reads back (the
    reference's reader layout) to the state within the format's 6
    significant digits."""
    from blaze.project import read_state_file
    g = mill
    s = device.Simulation(sim_info=g.sim_info, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                          dobj=g.dobj, n_d=g.n_d)
    st = g.init()
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    s.step(50)
    a = s.state()
    path = str(tmp_path / "state.dat")
    s.write_state(path, detail=3, sim_type=1, rev_number=1, revflag=0, time=50 * 1e-5,
                  steps_per_rev=272727, dt=1e-5)
    s.close()
    b = read_state_file(path, g.n, sim_type=1)
    np.testing.assert_array_equal(b["pid"], a["pid"])
    np.testing.assert_array_equal(b["type"], a["type"])
    for key in ("pos", "vel", "avel"):
        np.testing.assert_allclose(b[key], a[key], rtol=1e-5, atol=1e-30, err_msg=key)
