"""State files: the library's writer (blaze_write_state_arrays) against the
reference's own Output_SystemState (Input/FileIO.h:12-315) run on the same
arrays by oracle/_ref/refwriter, byte for byte: detail levels 1-5, spheres
and polyhedra, general / mill / silo / rotating-world-object headers,
particles removed from the run (P_ID -1) skipped.  CPU only."""
import ctypes
import os
import struct
import subprocess

import numpy as np
import pytest

from blaze import device
from blaze import types as T
from conftest import Golden

HERE = os.path.dirname(os.path.abspath(__file__))
REFWRITER = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "refwriter")

pytestmark = pytest.mark.skipif(not os.path.isfile(REFWRITER), reason="oracle/_ref not built")

CASES = [  # detail, sim_type, rotating, particle_type, revflag
    (1, 0, 0, 0, 0), (2, 0, 0, 0, 0), (3, 2, 0, 0, 0), (4, 1, 0, 0, 1), (3, 0, 1, 0, 0),
    (1, 1, 0, 1, 0), (2, 0, 0, 1, 0), (3, 1, 0, 1, 1), (4, 2, 0, 1, 0), (5, 0, 0, 1, 0),
]


def arrays(seed, n, n_p):
    rng = np.random.default_rng(seed)
    f = lambda *s: (rng.standard_normal(s) * rng.choice([1e-3, 1.0, 37.5, 1e4], size=s)).astype(np.float32)
    pid = rng.permutation(n).astype(np.int32)
    pid[rng.choice(n, 5, replace=False)] = -1
    return dict(pos=f(n, 3), quat=f(n, 4), vel=f(n, 3), avel=f(n, 3), acc=f(n, 3),
                type=rng.integers(0, n_p, n).astype(np.uint32), pid=pid)


@pytest.mark.parametrize("case", CASES)
def test_writer_matches_reference(case, tmp_path):
    detail, sim_type, rotating, ptype, revflag = case
    g = Golden("box_poly")
    n, n_p = 60, g.n_p
    a = arrays(sum(case) * 7 + detail, n, n_p)
    h = device.state_header(detail=detail, sim_type=sim_type, rotating_wobj=rotating,
                            particle_type=ptype, revflag=revflag, rev_number=3, num_rem=1234,
                            rot_steps=777, steps_per_rev=272727, time=1.23456789,
                            rot_angle=-6.2831853, energy=[873.66, 424.12, 251.27, 1.5, 2.5],
                            hatch_height=0.25, dt=1e-5)
    ours = tmp_path / "ours.dat"
    device.write_state_arrays(str(ours), h, a["pos"], a["vel"], a["avel"], a["acc"], a["type"],
                              a["pid"], quat=a["quat"], pobj=g.pobj, n_p=n_p)
    # the reference writer's input
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as fh:
        fh.write(struct.pack("<11i", n, detail, sim_type, rotating, ptype, revflag, 3, 1234, 777,
                             272727, n_p))
        fh.write(struct.pack("<2d", 1.23456789, -6.2831853))
        fh.write(np.array([873.66, 424.12, 251.27, 1.5, 2.5, 0.25, 1e-5], np.float32).tobytes())
        for key in ("pos", "quat", "vel", "avel", "acc", "type", "pid"):
            fh.write(np.ascontiguousarray(a[key]).tobytes())
        fh.write(bytes(g.pobj)[:ctypes.sizeof(T.POBJ) * n_p])
    run = tmp_path / "run"
    run.mkdir()
    subprocess.run([REFWRITER, str(inp), str(run)], check=True, capture_output=True)
    ref = tmp_path / "Results" / "P" / "W" / "SystemState1.23457.dat"
    assert ref.read_bytes() == ours.read_bytes()
