"""Named workload cases for timing and profiling the ensemble path and its
reverse mode on one GPU (the commands in the repository's profile summaries
run these).

    python softx-d-15-00085_b200/blaze/cases.py ens_step [STEPS]
        96 systems of the batched workload (1,442,352 spheres), skin 0.01 cm,
        blocks of 128, a 1,500-step pre-roll, then STEPS plain steps (30).
    python softx-d-15-00085_b200/blaze/cases.py adjoint [NSYS] [STEPS] [SEGMENT] [TAPE_BYTES]
        calibration ensemble of NSYS x 20,000 spheres (64), seeded initial
        velocities, reverse mode over STEPS steps (60) with checkpoints every
        SEGMENT (30), random cotangents of the final state.
    python softx-d-15-00085_b200/blaze/cases.py poly [N] [STEPS]
        the convex-polyhedra workload of bench.py at N particles (20,000),
        reference mode, STEPS plain steps (10).
"""
import os
import sys

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402

from blaze import autotune, calibrate, synth  # noqa: E402
from blaze import ensemble as E  # noqa: E402


def ens_step(steps=30):
    counts = synth.batched_counts(512, seed=3)[:96]
    rng = np.random.default_rng(3)
    S, W, p, r = synth.box_ensemble(counts, mus=rng.uniform(0.2, 0.8, 96),
                                    restitutions=rng.uniform(0.3, 0.9, 96), seed=3)
    S = autotune.regrid(S, 0.01, 0.2)
    pos, vel = autotune.preroll(S, W, p, r, None, 1500, law=E.LAW_LINEAR, dt=1e-5, max_nbr=32,
                                skin=0.01)
    e = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.01, use_graph=0, block=128)
    e.set_state(pos, r, vel)
    e.step(steps)
    status = e.sync()
    print("ens_step: n %d status %d rebuilds %d" % (e.n, status, e.num_rebuilds()))
    e.close()
    return status


def poly(n=20000, steps=10):
    """The convex-polyhedra bench workload at n particles, reference mode
    (contact list rebuilt every step), `steps` plain steps."""
    import tempfile
    from blaze import device
    with tempfile.TemporaryDirectory() as d:
        P, st = synth.poly_box_project(d, n=n)
    sim = device.Simulation(P)
    sim.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"], quat=st["quat"])
    sim.step(steps)
    status = sim.sync()
    print("poly: n %d status %d" % (n, status))
    sim.close()
    return status


def adjoint(nsys=64, steps=60, segment=30, tape_bytes=0):
    """The calibration ensemble (nsys x 20,000 spheres), `steps` steps with
    checkpoints every `segment`, the tape budget `tape_bytes` (0: one
    segment; -1: 90 % of the free device memory), forward and backward."""
    S, W, p, r = calibrate.calibration_ensemble(nsys=nsys, n=20000, seed=4)
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.02, use_graph=0)
    ens.set_state(p, r, calibrate.initial_velocity(len(p)))
    adj = E.Adjoint(ens, steps, segment, tape_bytes)
    status = adj.forward()
    st = ens.state()
    g = np.random.default_rng(0).normal(size=st["pos"].shape).astype(np.float32)
    adj.backward(g, g * 1e-2, None)
    print("adjoint: n %d status %d rebuilds %d" % (ens.n, status, ens.num_rebuilds()))
    adj.close()
    ens.close()
    return status


if __name__ == "__main__":
    name = sys.argv[1] if len(sys.argv) > 1 else "ens_step"
    args = [int(a) for a in sys.argv[2:]]
    rc = {"ens_step": ens_step, "adjoint": adjoint, "poly": poly}[name](*args)
    sys.exit(1 if rc else 0)
