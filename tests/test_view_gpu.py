"""The headless view buffer (blaze_device_view), the replacement of the
reference's OpenGL view: device pointers to the current positions and, for
polyhedra, orientations, read here through __cuda_array_interface__ (no
copy) and compared with the state the reference-facing getters return."""
import numpy as np
import pytest
import torch

from blaze import device, synth
from conftest import Golden

pytestmark = pytest.mark.gpu


class _DeviceArray:
    """A float32 (n, 4) device array at a raw pointer, for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n, 4), "typestr": "<f4", "data": (ptr, False),
                                         "version": 2}


def view(sim):
    pos, orn, n, _ = sim.device_view()
    p = torch.as_tensor(_DeviceArray(pos, n), device="cuda").cpu().numpy()
    q = None if orn is None else torch.as_tensor(_DeviceArray(orn, n), device="cuda").cpu().numpy()
    return p, q


def test_view_spheres(tmp_path):
    P, st = synth.box_project(str(tmp_path), n_side=(10, 10, 10))
    sim = device.Simulation(P, skin=0.02, use_graph=1)
    sim.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    sim.step(37)
    p, q = view(sim)
    s = sim.state()
    sim.close()
    assert q is None and s["status"] == 0
    np.testing.assert_array_equal(p[:, :3], s["pos"])
    np.testing.assert_array_equal(p[:, 3], np.float32(0.1))


def test_view_polyhedra_orientations():
    g = Golden("box_poly")
    sim = device.Simulation(sim_info=g.sim_info, wobj=g.wobj, n_w=g.n_w, pobj=g.pobj, n_p=g.n_p,
                            dobj=g.dobj, n_d=g.n_d, skin=0.05, use_graph=1)
    st = g.init()
    sim.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"], quat=st["quat"])
    for k in range(3):          # re-sorts in between switch the orientation copy
        sim.step(13)
        p, q = view(sim)
        s = sim.state()
        assert s["status"] == 0
        np.testing.assert_array_equal(q, s["quat"])
        # positions: centres of mass; the getters return pos - COM per type
        off = p[:, :3] - s["pos"]
        for t in np.unique(s["type"]):
            o = off[s["type"] == t]
            np.testing.assert_allclose(o, np.broadcast_to(o[0], o.shape), rtol=0, atol=1e-4)
    sim.close()
