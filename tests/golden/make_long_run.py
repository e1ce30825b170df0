"""Generate tests/golden/long_run.npz: long-horizon statistics of oracle A
(the reference's kernels compiled as host C++, oracle/_ref) that the GPU
tests compare the library's Verlet-skin path with.

  silo_sph90  Projects/2.Silo, world SPH_90, from its start file: the hatch
              opened at t = 0 as the headless driver does
              (main.cpp:1049-1055), then Silo_Stats' count of the particles
              above the hatch every 8,696 steps (main.cpp:253-280, 133-147;
              8,696 is the world file's Flow_counter value), 20 counts
              (1.74 s of discharge).
  box_c1      the Particles_Box plain configuration (10,000 spheres,
              r = 0.1 cm, in a 10 cm cube, falling from a jittered lattice):
              kinetic energy (translational + rotational) every 100 steps to
              12,000 steps, the dissipated-energy tallies at the same steps
              (the per-contact values summed in FP64, as the library sums
              them; box_edis_float_tally: the reference's own FP32
              accumulators, which lose the small late contributions), and
              the vertical solid-fraction profile at 2,000 and 12,000 steps.

Each case runs R_RUNS times: run 0 from the given state, the others with
every position coordinate moved by one unit in the last place, up or down at
random (seeded).  The spread across the runs is the reference's own
sensitivity to round-off over the horizon; the tests' bands are set from it.

Run from the repository root (needs the reference tree for the project files
and oracle/_ref built by `make -C oracle ref`):
    python tests/golden/make_long_run.py
"""
import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(REPO, "softx-d-15-00085_b200"), os.path.join(REPO, "oracle"),
          os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

R_RUNS = 4
SILO_FLOW_STEPS = 8696
SILO_LINES = 20
BOX_EVERY = 100
BOX_STEPS = 12000
BOX_PROFILE_AT = (2000, 12000)


def perturb(pos, run):
    """One-ulp moves of every coordinate (run 0: unchanged)."""
    if run == 0:
        return pos
    rng = np.random.default_rng(1000 + run)
    up = rng.integers(0, 2, size=pos.shape).astype(bool)
    return np.where(up, np.nextafter(pos, np.float32(np.inf)),
                    np.nextafter(pos, np.float32(-np.inf))).astype(np.float32)


def _silo(run, threads):
    from bindings import RefHost
    from conftest import Golden
    g = Golden("silo_sph90")
    st = g.init()
    R = RefHost().init(g.sim_info, g.wobj, g.n_w, g.pobj, g.n_p, g.dobj, g.n_d, threads=threads,
                       capture=False)
    R.set_state(perturb(st["pos"], run), st["vel"], st["avel"], st["type"], st["pid"])
    R.lib.refh_open_hatch(g.wobj, g.n_w - 1)
    h = float(g.wobj[g.n_w - 1].vertex[0].y)
    above = []
    for _ in range(SILO_LINES):
        assert R.step(SILO_FLOW_STEPS) == 0
        above.append(int((R.state()["pos"][:, 1] > h).sum()))
    return np.array(above, np.int32)


def _box(run, threads):
    from bindings import RefHost
    from blaze import synth
    import long_run_stats as S
    P, st = synth.box_project(tempfile.mkdtemp(prefix="box_c1_"))
    P.sim_info.EnergyCalc = True
    R = RefHost().init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d, threads=threads,
                       capture=False)
    R.set_state(perturb(st["pos"], run), st["vel"], st["avel"], st["type"], st["pid"])
    m, r = float(P.pobj[0].mass), float(P.pobj[0].radius)
    ke, edis, edis32, prof = [], [], [], []
    for k in range(BOX_EVERY, BOX_STEPS + 1, BOX_EVERY):
        assert R.step(BOX_EVERY) == 0
        s = R.state()
        ke.append(S.kinetic_energy(s["vel"], s["avel"], m, r))
        edis.append(R.energy64()[[0, 2]])
        edis32.append(np.asarray(R.energy(), np.float64)[[0, 2]])
        if k in BOX_PROFILE_AT:
            prof.append(S.solid_fraction_profile(s["pos"], r))
    return np.array(ke), np.array(edis), np.array(prof), np.array(edis32)


def _job(args):
    kind, run, threads = args
    return (kind, run, _silo(run, threads) if kind == "silo" else _box(run, threads))


def main():
    threads = max(1, (os.cpu_count() or 2) // R_RUNS)
    jobs = [(k, r, threads) for k in ("silo", "box") for r in range(R_RUNS)]
    with mp.get_context("spawn").Pool(R_RUNS) as pool:
        res = pool.map(_job, jobs)
    silo = np.stack([v for k, r, v in sorted(res, key=lambda x: x[1]) if k == "silo"])
    box = [v for k, r, v in sorted(res, key=lambda x: x[1]) if k == "box"]
    out = dict(silo_above=silo, silo_flow_steps=SILO_FLOW_STEPS, silo_n0=1950,
               box_every=BOX_EVERY, box_steps=BOX_STEPS,
               box_profile_at=np.array(BOX_PROFILE_AT),
               box_ke=np.stack([b[0] for b in box]), box_edis=np.stack([b[1] for b in box]),
               box_profile=np.stack([b[2] for b in box]),
               box_edis_float_tally=np.stack([b[3] for b in box]), runs=R_RUNS)
    path = os.path.join(HERE, "long_run.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")
    print("silo above per line (run 0):", silo[0].tolist())
    print("box KE every 1000 steps (run 0):", out["box_ke"][0][9::10].round(3).tolist())


if __name__ == "__main__":
    main()
