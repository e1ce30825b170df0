"""Convex polyhedra, CPU side: the committed fixture is what the reference's
own polyhedron kernels (oracle A, oracle/_ref) produce from its initial
state, checkpoint by checkpoint."""
import numpy as np
import pytest

import bindings

need_ref_lib = pytest.mark.skipif(not bindings.ref_available(), reason="oracle/_ref not built")

STATE_KEYS = ("pos", "quat", "vel", "avel", "type", "pid")
FORCE_KEYS = ("f_pp", "t_pp", "f_wall", "t_wall", "f_lift", "t_lift")


@need_ref_lib
def test_reference_replays_fixture(golden_poly):
    g = golden_poly
    R = bindings.RefHost()
    R.init(g.sim_info, g.wobj, g.n_w, g.pobj, g.n_p, g.dobj, g.n_d, threads=4, capture=True)
    R.set_cylinder_rotation(g.cyl_rot)
    s0 = g.init()
    R.set_state(s0["pos"], s0["vel"], s0["avel"], s0["type"], s0["pid"], quat=s0["quat"])
    done = 0
    for k in g.checkpoints:
        assert R.step(k - done) == 0
        done = k
        ref = g.at(k)
        st = R.state()
        for key in STATE_KEYS:
            np.testing.assert_array_equal(st[key], ref[key], err_msg="%s step %d" % (key, k))
        f = R.forces()
        for key in FORCE_KEYS:
            np.testing.assert_array_equal(f[key], ref[key], err_msg="%s step %d" % (key, k))
        nn, lst = R.nlist()
        np.testing.assert_array_equal(nn, ref["nn"])


def test_fixture_exercises_contacts(golden_poly):
    """The fixture is a useful parity case: polyhedron pairs in contact
    (torques), floor contacts, orientations that change every step."""
    g = golden_poly
    s1 = g.at(1)
    assert int((np.abs(s1["t_pp"]).sum(axis=1) > 0).sum()) > 0.3 * g.n
    assert int((np.abs(s1["f_wall"]).sum(axis=1) > 0).sum()) > 20
    if g.cyl_rot:  # drum wall contacts carry torque (end plates do not)
        assert int((np.abs(s1["t_wall"]).sum(axis=1) > 0).sum()) > 100
    if g.n_d:  # lifter contacts, with torque
        assert int((np.abs(s1["t_lift"]).sum(axis=1) > 0).sum()) > 5
    s0 = g.init()
    order0 = np.argsort(s0["pid"])
    order1 = np.argsort(s1["pid"])
    dq = np.abs(s1["quat"][order1] - s0["quat"][order0]).max(axis=1)
    assert np.all(dq > 0)
