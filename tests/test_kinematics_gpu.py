"""The mill driver's per-step moves of world and volume objects
(Processing_Mills.h) run on the device, against oracle A running the
reference's kernels with the same moves restated on the host
(oracle/ref_host/refhost_kernels.cpp), live on the GPU box:

* rotating world objects (Rotate_WObject_inc): the silo fixture's objects
  marked rotating, turned 2.3e-5 rad per step about a point of the silo's
  mid-plane, moving-surface law on (Rotating_WObject with drum rotation);
* a translating volume object (Translate_VolObject) beside the seven other
  lifters of the mill fixture turning with the drum.

Bar: positions, velocities, spins, P_ID and the moved objects' vertices,
normals, centroids and areas bit for bit after 1, 50 and 200 steps.
"""

import numpy as np
import pytest

import bindings
from blaze import device
from blaze import types as T
from conftest import Golden

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not bindings.ref_available(), reason="oracle/_ref not built")]

STEPS = (1, 49, 150)
STATE = ("pos", "vel", "avel", "pid")


def copies(g):
    si = T.SimulationInfo.from_buffer_copy(bytes(g.sim_info))
    wobj = (T.WOBJ * 8).from_buffer_copy(bytes(g.wobj))
    dobj = (T.DOBJ * 32).from_buffer_copy(bytes(g.dobj))
    return si, wobj, dobj


def faces(objs, n, kind):
    out = []
    for k in range(n):
        o = objs[k]
        nv = o.num_vertex
        out += [(v.x, v.y, v.z) for v in list(o.vertex)[:nv]]
        surf = o.surfaces if kind == "w" else o.faces
        ns = o.num_surfaces if kind == "w" else o.num_faces
        for f in range(ns):
            s = surf[f]
            out += [(s.normal.x, s.normal.y, s.normal.z), (s.centroid.x, s.centroid.y, s.centroid.z),
                    (s.area, 0.0, 0.0)]
    return np.array(out, np.float32)


def run_pair(g, si, wobj, dobj, setup_ref, setup_gpu, kind, n_obj):
    st = g.init()
    R = bindings.RefHost()
    R.init(si, wobj, g.n_w, g.pobj, g.n_p, dobj, g.n_d, threads=8, capture=False)
    R.set_cylinder_rotation(True)
    R.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    setup_ref(R)
    s = device.Simulation(sim_info=si, wobj=wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p, dobj=dobj,
                          n_d=g.n_d, use_graph=1)
    s.set_cylinder_rotation(True)
    s.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    setup_gpu(s)
    for chunk in STEPS:
        assert R.step(chunk) == 0
        s.step(chunk)
        a, b = s.state(), R.state()
        assert a["status"] == 0, device.decode_status(a["status"])
        for key in STATE:
            np.testing.assert_array_equal(a[key], b[key], err_msg=key)
        if kind == "w":
            fa, fb = faces(s.wobj(), n_obj, "w"), faces(R.wobj(g.n_w), n_obj, "w")
        else:
            fa, fb = faces(s.dobj(), n_obj, "d"), faces(R.dobj(g.n_d), n_obj, "d")
        np.testing.assert_array_equal(fa, fb)
    s.close()
    return fa


def test_rotating_world_objects():
    g = Golden("silo_sph90")
    si, wobj, dobj = copies(g)
    si.Rotating_WObject = True
    si.MillRotVel = -0.5
    for k in range(g.n_w):
        wobj[k].is_rotating = True
    v = np.array([[p.x, p.y] for k in range(g.n_w) for p in list(wobj[k].vertex)[:wobj[k].num_vertex]])
    ax, ay = [float(np.float32(x)) for x in v.mean(axis=0)]
    rad = float(np.float32(-2.3e-5))
    before = faces(wobj, g.n_w, "w")
    after = run_pair(g, si, wobj, dobj, lambda R: R.set_wobj_rotation(ax, ay, rad),
                     lambda s: s.set_wobj_rotation(ax, ay, rad), "w", g.n_w)
    assert np.any(after != before)


def test_translating_volume_object():
    g = Golden("mill_sph30")
    si, wobj, dobj = copies(g)
    d0 = dobj[0]
    d0.is_attached_DWorld = False
    d0.is_translating = True
    d0.velocity.x, d0.velocity.y, d0.velocity.z = 0.0, 40.0, 0.0
    r = float(wobj[0].cyl_geo.radius)
    rad = float(np.float32(-2.303834662598092e-05))

    def ref(R):
        R.set_dobj_rotation(r, r, rad)
        R.set_dobj_translation(0)

    def gpu(s):
        s.set_dobj_rotation(r, r, rad)
        s.set_dobj_translation(0)

    before = faces(dobj, g.n_d, "d")
    after = run_pair(g, si, wobj, dobj, ref, gpu, "d", g.n_d)
    assert np.any(after != before)
