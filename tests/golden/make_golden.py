"""Generate the golden fixtures under tests/golden/ from the reference's own
project files and the reference's own kernels (oracle A: the reference's
DEM kernels compiled as host C++, oracle/_ref/libblaze_refhost.so).

Run in a container that has the reference tree (its path is the first
argument, default /root/reference) after `make -C oracle ref`:

    python tests/golden/make_golden.py [/path/to/reference]

Each fixture is an .npz with
  wobj, pobj, dobj, sim_info   raw bytes of the boundary structs as this
                               project's parser builds them (checked field by
                               field against the reference's parser)
  n_w, n_p, n_d, cyl_rot       counts and the drum-rotation flag
  init_*                       the initial state read from the fixture file
  s{K}_*                       oracle A after K steps: pos, vel, avel, type,
                               pid, the force arrays of step K before
                               integration, and the contact list of step K
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "softx-d-15-00085_b200"))

from bindings import RefHost  # noqa: E402
import canon  # noqa: E402
from blaze.project import Project  # noqa: E402

CHECKPOINTS = (1, 2, 10, 100)

# (fixture name, project, world, drum rotation on)
FIXTURES = [
    ("silo_sph90", "2.Silo", "SPH_90", False),
    ("mill_sph30", "3.BallMill", "Mill_SPH30", True),
]


def make(ref_root, name, project, world, cyl_rot):
    projects = os.path.join(ref_root, "Projects")
    P = Project.load(projects, project, world)
    R = RefHost()
    rp, w, p, d = R.parse(projects, project, world)
    # the project-input mirror must agree with the reference's parser
    assert [canon.wobj(w[i]) for i in range(rp.n_w)] == [canon.wobj(P.wobj[i]) for i in range(P.n_w)]
    assert [canon.pobj_sphere(p[i], rp.n_p) for i in range(rp.n_p)] == \
        [canon.pobj_sphere(P.pobj[i], P.n_p) for i in range(P.n_p)]
    assert [canon.dobj(d[i]) for i in range(rp.n_d)] == [canon.dobj(P.dobj[i]) for i in range(P.n_d)]
    st = P.read_state()
    R.init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d, threads=4, capture=True)
    R.set_cylinder_rotation(cyl_rot)
    R.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    out = dict(
        wobj=np.frombuffer(bytes(P.wobj), np.uint8), pobj=np.frombuffer(bytes(P.pobj), np.uint8),
        dobj=np.frombuffer(bytes(P.dobj), np.uint8),
        sim_info=np.frombuffer(bytes(P.sim_info), np.uint8),
        n_w=P.n_w, n_p=P.n_p, n_d=P.n_d, cyl_rot=int(cyl_rot),
        init_pos=st["pos"], init_vel=st["vel"], init_avel=st["avel"], init_type=st["type"],
        init_pid=st["pid"], source="%s/World/%s.World" % (project, world))
    done = 0
    for k in CHECKPOINTS:
        rc = R.step(k - done)
        assert rc == 0, rc
        done = k
        s = R.state()
        f = R.forces()
        nn, lst = R.nlist()
        for key in ("pos", "vel", "avel", "type", "pid"):
            out["s%d_%s" % (k, key)] = s[key]
        for key, v in f.items():
            out["s%d_%s" % (k, key)] = v
        out["s%d_nn" % k] = nn
        out["s%d_list" % k] = lst[:, :max(1, int(nn.max()))]
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    for name, project, world, rot in FIXTURES:
        make(ref_root, name, project, world, rot)


if __name__ == "__main__":
    main()
