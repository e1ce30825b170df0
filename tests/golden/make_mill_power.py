"""Generate tests/golden/mill_power.npz: the ball-mill power known answer.

The reference's ReadMe for its ball mill (Projects/3.BallMill/ReadMe.txt:5-6)
states the values `Mill_SPH30` must give after the first revolution:
  time 2.72727  Power: Total = 625.98  Particle 319.724  Lifter 156.378
  Drum 149.878
(W: energy dissipated in particle-particle, lifter and drum contacts over the
revolution, divided by its duration; main.cpp:53-70).  This script runs the
same revolution on oracle A (the reference's own kernels compiled for the
host, oracle/_ref) with the mill driver's per-step lifter turn
(Processing_Mills.h:4-75, main.cpp:113-124, restated in
oracle/ref_host/refhost_kernels.cpp) and the drum rotating, one host thread
so the FP32 tallies add in particle order (and an FP64 sum of the same
values beside them), and stores the structs, the
initial state, the mill constants, checkpoints of the state and tallies and
the published numbers.

Run in a container that has the reference tree, after `make -C oracle ref`:

    python tests/golden/make_mill_power.py [/path/to/reference]

About 70 s of CPU.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "softx-d-15-00085_b200"))

from bindings import RefHost  # noqa: E402
from blaze.project import Project  # noqa: E402

PUBLISHED = {"time": 2.72727, "total": 625.98, "particle": 319.724, "lifter": 156.378,
             "drum": 149.878}


def main(ref_root):
    P = Project.load(os.path.join(ref_root, "Projects"), "3.BallMill", "Mill_SPH30")
    nspr = int(P.mill.Num_Steps_PerRev)
    rad = np.float32(P.mill.RadPerStep)
    about = np.float32(P.wobj[0].cyl_geo.radius)
    st = P.read_state()
    R = RefHost()
    R.init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d, threads=1, capture=False)
    R.set_cylinder_rotation(True)
    R.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    R.reset_energy()
    R.set_dobj_rotation(about, about, rad)
    out = dict(
        wobj=np.frombuffer(bytes(P.wobj), np.uint8), pobj=np.frombuffer(bytes(P.pobj), np.uint8),
        dobj=np.frombuffer(bytes(P.dobj), np.uint8),
        sim_info=np.frombuffer(bytes(P.sim_info), np.uint8),
        n_w=P.n_w, n_p=P.n_p, n_d=P.n_d, cyl_rot=1,
        init_pos=st["pos"], init_vel=st["vel"], init_avel=st["avel"], init_type=st["type"],
        init_pid=st["pid"], steps_per_rev=nspr, rad_per_step=rad, about=about,
        dt=np.float32(P.sim_info.InitalDelta_t),
        published=np.array([PUBLISHED[k] for k in ("total", "particle", "lifter", "drum")]),
        source="3.BallMill/World/Mill_SPH30.World")
    checkpoints = [1, 100, 10000, nspr]
    done = 0
    for k in checkpoints:
        rc = R.step(k - done)
        assert rc == 0, rc
        done = k
        s = R.state()
        for key in ("pos", "vel", "avel", "pid"):
            out["s%d_%s" % (k, key)] = s[key]
        out["s%d_energy" % k] = R.energy()
        out["s%d_energy64" % k] = R.energy64()
        d = R.dobj(P.n_d)
        out["s%d_lifter_vertex" % k] = np.array(
            [[[d[q].vertex[v].x, d[q].vertex[v].y, d[q].vertex[v].z] for v in range(8)]
             for q in range(P.n_d)], np.float32)
        print("step %d energy %s" % (k, out["s%d_energy" % k]), flush=True)
    out["checkpoints"] = np.array(checkpoints)
    T = nspr * float(np.float32(P.sim_info.InitalDelta_t))
    for key in ("energy", "energy64"):
        e = out["s%d_%s" % (nspr, key)].astype(np.float64)
        print("oracle A power after one revolution (%s tallies): total %.3f particle %.3f "
              "lifter %.3f drum %.3f" % (key, e.sum() / T, e[0] / T, e[1] / T, e[2] / T))
    np.savez_compressed(os.path.join(HERE, "mill_power.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "BLAZE_REFERENCE", os.path.join(os.path.dirname(REPO), "reference")))
