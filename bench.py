"""Throughput of the DEM step on the silo-discharge workload (1,000,000
polydisperse spheres), reported as particle-steps/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl blaze|reference]

One process per GPU (torchrun for N > 1).  The DEM step does not shard: each
rank runs an independent replica of the workload (weak scaling, no
data-path collective); the barrier and the max-over-ranks time reduction use
the process group only.

Workload: the silo discharge configuration in its reference-law form (the
form the reference's own code can run): a 25 cm barrel over a 30 degree
hopper to a 6 cm outlet as 7 sector world objects of planar quads (the
reference's own silo is built of planar faces), 1,000,000 spheres with
radius uniform in [0.2, 0.4] cm quantised to 6 particle objects, density
2600 kg/m^3, linear spring-dashpot kn = 1e5 kg/s^2, restitution 0.6,
mu 0.5, dt = 5e-6 s, FP32; synthetic seeded packing (no dataset exists),
settled with the hatch closed before the hatch opens and the timing starts.
The full form (Hertz-Mindlin, 4,096-triangle hopper, which the reference
cannot run) is the line's `silo_full` entry, and `--silo-full-only` prints
it alone.

Timed region (value): K steps enqueued through the handle API on device-
resident state, bracketed by CUDA events on the library's stream.
e2e: the same K steps through the reference-facing C ABI with host
buffers: every step uploads the full particle state from pinned host memory
(Device_Set_System_State), runs Device_DEM_UpdateSim and reads the state
back (Device_Get_System_State).
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "softx-d-15-00085_b200")
sys.path.insert(0, PKG)

METRIC = "particle-steps/s at 1M spheres"
UNIT = "particle-steps/s"
B_ALG = 96  # bytes per particle-step of the fused step: 3 float4 streams read + written


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="blaze", choices=["blaze", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--skin", type=float, default=0.16,
                    help="Verlet skin, cm (0 = reference mode); 0.16 was the fastest of "
                         "0.02-0.16 on the settled discharge")
    ap.add_argument("--law", default="fast", choices=["exact", "fast"],
                    help="particle-particle law of the timed steps: the reference's arithmetic "
                         "bit for bit, or its contracted form (forces within 1e-5 relative)")
    ap.add_argument("--max-nbr", type=int, default=32)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--settle-steps", type=int, default=48000,
                    help="untimed settling of the generated packing with the hatch closed "
                         "before the discharge is timed (48,000 steps: the bed's contacts per "
                         "particle have stopped rising)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-ensemble leg (512 box-settling systems)")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the reverse-mode leg (64 x 20,000-sphere calibration ensemble)")
    ap.add_argument("--adjoint-steps", type=int, default=3000)
    ap.add_argument("--batched-steps", type=int, default=2000,
                    help="timed steps of the batched leg (the workload's 2,000 settling steps)")
    ap.add_argument("--no-silo-full", action="store_true",
                    help="skip the full silo form (Hertz-Mindlin, 4,096-triangle hopper, 1M)")
    ap.add_argument("--silo-full-steps", type=int, default=10000,
                    help="timed steps of the full silo form (the workload's 10,000 steps)")
    ap.add_argument("--silo-full-only", action="store_true",
                    help="run only the full silo form and print its object")
    ap.add_argument("--no-poly", action="store_true",
                    help="skip the convex-polyhedra leg (100,000 polyhedra in a box)")
    ap.add_argument("--poly-steps", type=int, default=500)
    ap.add_argument("--no-mill", action="store_true", help="skip the ball-mill leg")
    ap.add_argument("--no-c1", action="store_true", help="skip the C1 box leg")
    ap.add_argument("--no-mill-mesh", action="store_true",
                    help="skip the turning-mesh ball-mill leg (ensemble path)")
    ap.add_argument("--no-mill-mixed", action="store_true",
                    help="skip the mixed-charge ball-mill leg (spheres + polyhedral rocks)")
    ap.add_argument("--mill-mixed-only", action="store_true",
                    help="run only the mixed-charge ball-mill leg and print its object")
    ap.add_argument("--mill-steps", type=int, default=5000)
    ap.add_argument("--mill-only", action="store_true",
                    help="print only the ball-mill leg's JSON line")
    ap.add_argument("--poly-only", action="store_true",
                    help="run only the convex-polyhedra leg and print its object")
    ap.add_argument("--case", nargs="+", metavar=("NAME", "ARG"),
                    help="run one named workload case for profiling (no timing line): "
                         "ens_step [STEPS], adjoint [NSYS STEPS SEGMENT TAPE_BYTES], "
                         "poly [N STEPS], silo_settled [N SETTLE STEPS FAST SKIN_UM]; see case_*")
    return ap.parse_args()


def case_ens_step(steps=30):
    """96 systems of the batched workload (1,442,352 spheres), skin 0.01 cm,
    blocks of 128, a 1,500-step pre-roll, then `steps` plain steps."""
    from blaze import autotune, synth
    from blaze import ensemble as E
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


def case_poly(n=20000, steps=10):
    """The convex-polyhedra workload of poly_leg at n particles, reference
    mode (contact list rebuilt every step), `steps` plain steps."""
    from blaze import device, synth
    with tempfile.TemporaryDirectory() as d:
        P, st = synth.poly_box_project(d, n=n, spacing=POLY_SPACING, jitter=POLY_JITTER)
    sim = device.Simulation(P)
    sim.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"], quat=st["quat"])
    sim.step(steps)
    status = sim.sync()
    print("poly: n %d status %d" % (n, status))
    sim.close()
    return status


def case_adjoint(nsys=64, steps=60, segment=30, tape_bytes=0):
    """The calibration ensemble (nsys x 20,000 spheres), `steps` steps with
    checkpoints every `segment`, the tape budget `tape_bytes` (0: one
    segment; -1: 96 % of the free device memory), forward and backward with
    random cotangents of the final state."""
    from blaze import calibrate
    from blaze import ensemble as E
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


def case_silo_settled(n=1_000_000, settle=48000, steps=8, fast=1, skin_um=1600):
    """The headline silo workload from its settled bed: n spheres settled
    `settle` steps with the hatch closed and the headline's 0.16 cm skin
    (cached under /tmp on the first run: the same command line run again
    loads the cache, so a profiler sees only `steps` plain steps of the
    discharge), hatch open, contracted law when `fast`, then skin
    skin_um / 1e4 cm (0: the reference mode, a re-sort every step)."""
    from blaze import device, synth
    skin = skin_um * 1e-4
    cache = os.path.join(tempfile.gettempdir(), "blaze_silo_settled_%d_%d.npz" % (n, settle))
    with tempfile.TemporaryDirectory() as d:
        P, st0 = synth.silo_project(d, n=n)
    sim = device.Simulation(P, skin=0.16, max_nbr=32, use_graph=1)
    if os.path.isfile(cache):
        z = np.load(cache)
        sim.set_state(z["pos"], z["vel"], z["avel"], z["type"], z["pid"])
    else:
        sim.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
        sim.step(settle)
        s = sim.state()
        np.savez(cache, **{k: s[k] for k in ("pos", "vel", "avel", "type", "pid")})
    sim.open_hatch()
    # plain stepping: a profiler cannot see kernels inside graphs with
    # conditional nodes
    sim.set_options(skin=skin, max_nbr=32, use_graph=0, fast_law=int(fast))
    sim.step(steps)
    status = sim.sync()
    print("silo_settled: n %d status %d" % (n, status))
    sim.close()
    return status


CASES = {"ens_step": case_ens_step, "adjoint": case_adjoint, "poly": case_poly,
         "silo_settled": case_silo_settled}


def contacts_per_particle(sim):
    """Mean overlapping neighbours per particle in the current list (host)."""
    from blaze.device import device_array
    nn, lst = sim.nlist()
    pos4 = device_array(sim.device_state()[0], len(nn), 4).cpu().numpy()
    r = pos4[:, 3].astype(np.float64)
    p = pos4[:, :3].astype(np.float64)
    c = 0
    for k in range(lst.shape[1]):
        ok = nn > k
        if not ok.any():
            break
        j = lst[ok, k].astype(np.int64)
        c += int((np.linalg.norm(p[ok] - p[j], axis=1) < r[ok] + r[j]).sum())
    return c / max(len(nn), 1)


def make_workload(root, n):
    from blaze import synth
    return synth.silo_project(root, n=n)


def config(args):
    return {"workload": "silo_discharge_reference_law", "particles": args.n,
            "radius_cm": [0.2, 0.4], "radius_bins": 6, "hopper_faces": 42,
            "law": "linear spring-dashpot kn=1e5 e=0.6 mu=0.5", "dt_s": 5e-6,
            "skin_cm": args.skin, "max_nbr": args.max_nbr,
            "l2": "inputs larger than L2 (state 3x48 MB + neighbour slots %d MB per step)"
                  % (args.n * args.max_nbr * 4 // 1000000),
            "parallelism": "replicas", "global_particles": args.n * args.gpus}


def peak_hbm():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the fused step kernel from the committed ncu
    summary (profiles/k_step_silo.md, line 'traffic_bytes_per_launch: X'
    with the particle count it was measured at), scaled to this N."""
    path = os.path.join(REPO, "profiles", "k_step_silo.md")
    try:
        vals = {}
        for line in open(path):
            if ":" in line:
                k, v = line.split(":", 1)
                vals[k.strip().strip("-* ")] = v.strip()
        return float(vals["traffic_bytes_per_launch"]), int(vals["particles"])
    except Exception:
        return None, None


class ClockSampler:
    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + q,
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


SEQ_SAMPLE = 64   # systems timed one at a time for the sequential comparator


def batched_leg(steps, warmup):
    """The batched ensemble: 512 independent box-settling systems, particle
    counts log-uniform in [2,000, 50,000] (seed 3), radii uniform in
    [0.1, 0.2] cm, boxes sized to a 0.55 solid fraction, per-system mu in
    [0.2, 0.8] and restitution in [0.3, 0.9], linear spring-dashpot with
    tangential history (kn = 1e5, kt = 2/7 kn), dt = 1e-5 s, skin and block
    size from the autotuner.
    The timed region is the whole settling run from rest (2,000 steps by
    default), re-sorts included, timed with graph stepping and with
    persistent stepping (use_graph 2); the faster is the value.  Compared with plain solves of single
    systems (same kernels and settings, one system per launch sequence): a
    seeded random sample of SEQ_SAMPLE of the 512 systems, each timed over
    the same steps from the same start; the sequential time of all 512 is
    512 x the sample's mean (the sum's unbiased estimate), with the
    sample's standard error scaled alike."""
    import torch
    from blaze import autotune, synth
    from blaze import ensemble as E
    counts = synth.batched_counts(512, seed=3)
    rng = np.random.default_rng(3)
    mus = rng.uniform(0.2, 0.8, len(counts))
    rests = rng.uniform(0.3, 0.9, len(counts))
    S, W, p, r = synth.box_ensemble(counts, mus=mus, restitutions=rests, seed=3)
    best, trials = autotune.tune(S, W, p, r, steps=200, warmup=max(3, warmup), preroll_steps=600)
    opts = dict(law=E.LAW_LINEAR, dt=1e-5, skin=best["skin"], use_graph=1, block=best["block"])
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    modes = {}
    # graph stepping (a conditional node and a step kernel per step) and
    # persistent stepping (one cooperative kernel between re-sorts, a grid
    # barrier per step); the faster is the leg's value
    for name, ug in (("graph", 1), ("persistent", 2)):
        ens = E.Ensemble(best["systems"], W, **dict(opts, use_graph=ug))
        ens.set_state(p, r)
        ens.step(max(3, warmup))
        ens.sync()
        stream = torch.cuda.ExternalStream(ens.device_state()[3])
        rb0 = ens.num_rebuilds()
        a.record(stream)
        ens.step(steps)
        b.record(stream)
        b.synchronize()
        ms_m = a.elapsed_time(b) / steps
        rb = ens.num_rebuilds() - rb0
        modes[name] = {"ms_per_step": ms_m, "rebuilds": rb, "status": ens.sync(),
                       "gpu_launches": ens.last_launches() + rb * ens.rebuild_kernels(),
                       "value": ens.n / (ms_m * 1e-3)}
        n = ens.n
        ens.close()
    mode = min(modes, key=lambda k: modes[k]["ms_per_step"])
    ms = modes[mode]["ms_per_step"]
    rebuilds = modes[mode]["rebuilds"]
    launches = modes[mode]["gpu_launches"]
    status = modes["graph"]["status"] | modes["persistent"]["status"]
    # single systems, one after another: a seeded random sample
    off = np.concatenate([[0], np.cumsum(counts)])
    pick = np.sort(np.random.default_rng(11).choice(len(counts), SEQ_SAMPLE, replace=False))
    single = []
    for s_ in pick:
        Ss = E.System.from_buffer_copy(bytes(best["systems"][s_]))
        Ss.wall0 = 0
        e1 = E.Ensemble([Ss], W[S[s_].wall0:S[s_].wall0 + 6], **opts)
        e1.set_state(p[off[s_]:off[s_ + 1]], r[off[s_]:off[s_ + 1]])
        e1.step(max(3, warmup))
        e1.sync()
        st1 = torch.cuda.ExternalStream(e1.device_state()[3])
        a.record(st1)
        e1.step(steps)
        b.record(st1)
        b.synchronize()
        single.append((int(counts[s_]), a.elapsed_time(b) / steps))
        e1.close()
    ts = np.array([x[1] for x in single])
    seq_ms = float(len(counts) * ts.mean())
    seq_se = float(len(counts) * ts.std(ddof=1) / np.sqrt(len(ts)))
    return {"workload": "512 box-settling systems, N log-uniform in [2000, 50000], "
                        "linear spring-dashpot + tangential history, dt 1e-5 s",
            "particles": int(n), "systems": len(counts), "value": n / (ms * 1e-3),
            "unit": UNIT, "ms_per_step": ms, "steps": steps, "rebuilds": rebuilds,
            "gpu_launches": launches, "status": status,
            "autotuned": {"skin_cm": best["skin"], "cell_cm": best["cell"],
                          "block": best["block"],
                          "trials": [[t[0], t[1], round(t[2], 4), t[3]] for t in trials]},
            "stepping": mode, "modes": modes,
            "sequential_plain_ms_per_step": seq_ms, "vs_sequential_plain": seq_ms / ms,
            "sequential_plain_stderr_ms": seq_se,
            "sequential_sample": "%d of %d systems (seeded random), each timed over %d steps"
                                 % (len(single), len(counts), steps),
            "single_samples": [[n_, round(t_, 5)] for n_, t_ in single]}


WINDOW = 50   # steps of the windowed reverse sweep (blaze_ens_adj_backward_window)


def adjoint_leg(steps, segment=100):
    """Reverse mode on the calibration ensemble: 64 systems x 20,000 spheres
    (radii uniform in [0.1, 0.2] cm, seed 4) settling in 5 cm square-base
    boxes, linear law with tangential history, dt = 1e-5 s, seeded initial
    velocities (30 cm/s spread, 50 cm/s down) so contacts start at once.
    Timed with CUDA events on the ensemble's stream over `steps` steps: the
    plain forward (CUDA graphs, no tape), the checkpointing forward
    (blaze_ens_adj_forward: a checkpoint per segment, and the trailing
    segments that fit recorded into a tape of 96 % of the free HBM) and the
    backward (blaze_ens_adj_backward: recomputation of the segments the tape
    does not hold + reverse kernels), with the
    cotangents of the calibration loss (bed height + 32-bin side-wall force
    profile against targets from mu = 0.45, e = 0.55, kn = 8e4) already on
    the host.  The whole autograd call (torch conversions included) is
    reported beside it."""
    import torch
    from blaze import calibrate as CAL
    from blaze import ensemble as E
    S, W, p, r = CAL.calibration_ensemble(nsys=64, n=20000, seed=4)
    n = len(p)
    vinit = CAL.initial_velocity(n).astype(np.float32)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)

    def timed(stream, fn):
        a.record(stream)
        out = fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b), out

    plain = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=1e-5, skin=0.02, use_graph=1)
    plain.set_state(p, r, vinit)
    plain.step(8)
    plain.sync()
    st1 = torch.cuda.ExternalStream(plain.device_state()[3])
    fwd_ms = timed(st1, lambda: plain.step(steps))[0] / steps
    plain.close()
    run = CAL.Runner(S, W, p, r, steps, segment, tape_bytes=-1)
    st2 = torch.cuda.ExternalStream(run.ens.device_state()[3])
    vt = torch.tensor(vinit.astype(np.float64))
    hidden = torch.tensor([[8e4, 0.55, 0.45, 0.45]] * len(S), dtype=torch.float64)
    with torch.no_grad():
        pos, vel = CAL.EnsembleRun.apply(hidden, vt, run)   # also builds the graphs
        target = CAL.observables(pos, vel, hidden, S, r)
    guess = np.array([[1e5, 0.5, 0.4, 0.4]] * len(S))
    params = torch.tensor(guess, requires_grad=True)
    v0 = vt.clone().requires_grad_(True)
    t0 = time.perf_counter()
    pos, vel = CAL.EnsembleRun.apply(params, v0, run)
    loss = CAL.loss_fn(pos, vel, params, S, r, target)
    loss.backward()
    autograd_s = time.perf_counter() - t0
    g = params.grad.numpy()
    gv0 = v0.grad.numpy()
    # device-side phases alone, same run, cotangents prepared beforehand
    pos_t = pos.detach().clone().requires_grad_(True)
    vel_t = vel.detach().clone().requires_grad_(True)
    CAL.loss_fn(pos_t, vel_t, params.detach(), S, r, target).backward()
    run.ens.set_params(CAL.with_params(S, guess))
    run.ens.set_state(p, r, vinit)
    ck_ms, status = timed(st2, run.adj.forward)
    arena_bytes, on_tape, pool_max = run.adj.tape_info()
    pid = run.ens.state()["pid"]
    gx = pos_t.grad.numpy()[pid].astype(np.float32)
    gv = vel_t.grad.numpy()[pid].astype(np.float32)
    bwd_ms = timed(st2, lambda: run.adj.backward(gx, gv, None))[0]
    restore_ms, record_ms, reverse_ms = run.adj.profile()
    # the calibration's gradient over the last WINDOW steps (truncated
    # backpropagation, the harness's remedy for the chaotic growth)
    run.window = WINDOW
    params_w = torch.tensor(guess, requires_grad=True)
    pos, vel = CAL.EnsembleRun.apply(params_w, vt.clone(), run)
    CAL.loss_fn(pos, vel, params_w, S, r, target).backward()
    gw = params_w.grad.numpy()
    run.ens.set_params(CAL.with_params(S, guess))
    run.ens.set_state(p, r, vinit)
    run.adj.forward()
    win_ms = timed(st2, lambda: run.adj.backward(gx, gv, None, window=WINDOW))[0]
    run.close()
    return {"workload": "64 box-settling systems x 20,000 spheres, linear law + tangential "
                        "history, dt 1e-5 s; loss: bed height + 32-bin side-wall force profile",
            "particles": n, "steps": steps, "checkpoint_every": segment, "status": status,
            "forward_ms_per_step": fwd_ms,
            "forward_with_checkpoints_ms_per_step": ck_ms / steps,
            "backward_ms_per_step": bwd_ms / steps,
            "adjoint_vs_forward": (ck_ms + bwd_ms) / steps / fwd_ms,
            "backward_vs_forward": bwd_ms / steps / fwd_ms,
            "tape": {"arena_gb": arena_bytes / 1e9, "segments": -(-steps // segment),
                     "segments_recorded_by_forward": on_tape,
                     "max_pool_gb_per_segment": pool_max / 1e9},
            "backward_phases_ms_per_step": {"restore": restore_ms / steps,
                                            "record": record_ms / steps,
                                            "reverse": reverse_ms / steps},
            "autograd_call_s": autograd_s,
            "loss": float(loss.item()),
            # the discrete adjoint of this flow grows about 5 % per step (the
            # flow is chaotic), so over 3,000 steps the full sweep's FP32
            # cotangents overflow: reported, not hidden; the windowed sweep
            # is the harness's gradient
            "grad": {"finite_fraction_params": float(np.isfinite(g).mean()),
                     "finite_fraction_v0": float(np.isfinite(gv0).mean()),
                     "max_abs_finite_v0": float(np.abs(gv0[np.isfinite(gv0)]).max())
                     if np.isfinite(gv0).any() else None},
            "grad_windowed": {"window": WINDOW,
                              "finite_fraction_params": float(np.isfinite(gw).mean()),
                              "mean_over_systems": {k: float(gw[:, j].mean()) for j, k in
                                                    enumerate(CAL.PARAMS)},
                              "backward_ms": win_ms}}


POLY_SPACING, POLY_JITTER = 0.99, 0.005   # cm


def poly_leg(steps, warmup, n=100_000, cpu_seconds=15.0, skin=0.05, want_cpu=True):
    """Convex polyhedra on the reference path: 100,000 particles (the
    polyhedron count of the mill configuration) in a closed box, a third
    each dodecahedra, cubes and hexagonal prisms of circumradius 0.5 cm on a
    0.99 cm lattice jittered by +-0.005 cm (bounding spheres of lattice
    neighbours overlap, so vertex contacts exist from the first step, while
    no initial penetration reaches the 0.05 r at which the reference's
    polyhedron kernel starts to clamp, DEM_Kernels_Compute.cuh:917-950),
    random orientations,
    velocities N(0, 10 cm/s), spins N(0, 20 rad/s), linear law kn = 1e5,
    e = 0.5, mu = 0.4, dt = 1e-5 s, rotation on.  GPU: CUDA graphs with a
    `skin` Verlet list on the bounding spheres (value) and the reference's
    rebuild-every-step mode (reference_mode_value).  CPU: the reference's own
    polyhedron kernels (oracle/_ref) on all host threads, reference mode, a
    bounded sample of whole steps from the state the GPU reached after its
    timed steps (the same contacts), with the count of the kernel's
    penetration-clamp warnings."""
    import torch
    from blaze import device, synth
    with tempfile.TemporaryDirectory() as d:
        P, st = synth.poly_box_project(d, n=n, spacing=POLY_SPACING, jitter=POLY_JITTER)
    sim = device.Simulation(P, skin=skin, use_graph=1)
    sim.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"], quat=st["quat"])
    sim.prepare_graphs()
    sim.step(max(16, -(-warmup // 8) * 8))
    status = sim.sync()
    stream = torch.cuda.ExternalStream(sim.device_state()[3])
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    rb0 = sim.num_rebuilds()
    a.record(stream)
    sim.step(steps)
    b.record(stream)
    fixed = sim.last_launches()
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    rebuilds = sim.num_rebuilds() - rb0
    launches = fixed + rebuilds * sim.rebuild_kernels()
    status |= sim.sync()
    st_timed = sim.state()
    sim.set_profile(True)
    sim.step(min(steps, 100))
    ms_rebuild, ms_step, nprof = sim.profile()
    sim.set_profile(False)
    sim.set_options(skin=0.0, use_graph=1)
    sim.step(3)
    sim.sync()
    kref = min(steps, 200)
    a.record(stream)
    sim.step(kref)
    b.record(stream)
    b.synchronize()
    ref_ms = a.elapsed_time(b) / kref
    status |= sim.sync()
    sim.close()
    out = {"workload": "100,000 convex polyhedra (dodecahedra, cubes, hexagonal prisms, "
                       "circumradius 0.5 cm) in contact in a closed box, linear law kn=1e5 "
                       "e=0.5 mu=0.4, dt 1e-5 s, rotation on",
           "particles": n, "value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
           "steps": steps, "skin_cm": skin, "rebuilds": rebuilds, "gpu_launches": launches,
           "step_kernels_ms": ms_step / max(nprof, 1),
           "rebuild_ms_per_step": ms_rebuild / max(nprof, 1),
           "reference_mode_value": n / (ref_ms * 1e-3), "reference_mode_ms_per_step": ref_ms,
           "status": device.decode_status(status)}
    if want_cpu:
        cb = cpu_reference_rate(P, st_timed, cpu_seconds, hatch=False)
        out["cpu_baseline"] = cb
        if cb:
            cb["sample"] += ", from the state after the GPU's timed steps"
            out["vs_cpu_reference"] = out["value"] / cb["value"]
            out["reference_mode_vs_cpu_reference"] = out["reference_mode_value"] / cb["value"]
    return out


def mill_mesh_leg(steps=5000, warmup=20, n=100_000, settle=60000, skin=0.04):
    """The ball mill with its drum and lifters as a turning mesh of 16,384
    triangles and two end plates turning in place (ensemble path; the
    reference has no triangle walls): drum
    r = 50 cm, L = 30 cm, 8 lifters 4 x 4 cm, 30 rpm, n steel spheres
    r ~ U[0.3, 0.6] cm, linear law with tangential history kn = 1e6,
    e = 0.4, mu = 0.6, dt = 2e-6 s.  The charge, packed inside the lifter
    ring, runs `settle` untimed steps with the drum turning (0.12 s), then
    `steps` graph steps are timed with CUDA events."""
    import torch
    from blaze import synth
    from blaze import ensemble as E
    S, W, p, r = synth.drum_mesh_ensemble(n=n, skin=skin)
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=2e-6, skin=skin, use_graph=1)
    ens.set_state(p, r)
    ens.step(settle + max(3, warmup))
    ens.sync()
    stream = torch.cuda.ExternalStream(ens.device_state()[3])
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    rb0 = ens.num_rebuilds()
    a.record(stream)
    ens.step(steps)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    rebuilds = ens.num_rebuilds() - rb0
    launches = ens.last_launches() + rebuilds * ens.rebuild_kernels()
    st = ens.state()
    ens.close()
    x, y = st["pos"][:, 0].astype(np.float64), st["pos"][:, 1].astype(np.float64)
    # tangential velocity in the drum's sense of turn (clockwise seen from +z)
    vt = -(x * st["vel"][:, 1] - y * st["vel"][:, 0]) / np.maximum(np.hypot(x, y), 1e-9)
    return {"workload": "ball mill, drum and lifters as a turning mesh of %d triangles, 30 rpm, "
                        "%d steel spheres r 0.3-0.6 cm, linear law + tangential history kn 1e6 "
                        "e 0.4 mu 0.6, dt 2e-6 s" % (int(S[0].ntris), n),
            "particles": n, "triangles": int(S[0].ntris), "value": n / (ms * 1e-3), "unit": UNIT,
            "ms_per_step": ms, "steps": steps, "settle_steps": settle, "skin_cm": skin,
            "rebuilds": rebuilds, "gpu_launches": launches, "status": st["status"],
            "charge_mean_tangential_velocity_cm_s": float(vt.mean())}


def mill_mixed_leg(steps=5000, warmup=20, n_spheres=100_000, n_rocks=5_000, settle=60000,
                   skin=0.04, block=256, cpu_seconds=10.0, want_cpu=True):
    """The ball mill's mixed charge (ensemble path; the reference runs
    spheres or polyhedra, never both): the turning drum of mill_mesh_leg with
    n_spheres steel balls r ~ U[0.3, 0.6] cm and n_rocks rocks (convex hulls
    of 8-16 points on spheres of radius 0.5-1 cm, seed 2, density 2700
    kg/m^3): the configuration's 2,000,000 : 100,000 count ratio at the
    charge the drum holds.  Linear law with tangential history kn = 1e6,
    e = 0.4, mu = 0.6, dt = 2e-6 s, 30 rpm.  `settle` untimed steps with the
    drum turning, then `steps` graph steps timed with CUDA events.  CPU: the
    reference cannot run the charge, so the baseline is the C restatement
    of the same step (oracle/ens_oracle.c, FP32, one host thread, kind
    "port"), a bounded sample of whole steps from the GPU's state after its
    timed steps (histories start empty there)."""
    import torch
    from blaze import synth
    from blaze import ensemble as E
    S, W, p, r, sh, so, q = synth.mill_mixed_ensemble(n_spheres=n_spheres, n_rocks=n_rocks,
                                                      skin=skin)
    n = len(p)
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=2e-6, skin=skin, use_graph=1, block=block)
    ens.set_state(p, r)
    ens.set_polyhedra(sh, so, q)
    ens.step(settle + max(3, warmup))
    ens.sync()
    stream = torch.cuda.ExternalStream(ens.device_state()[3])
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    rb0 = ens.num_rebuilds()
    a.record(stream)
    ens.step(steps)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    rebuilds = ens.num_rebuilds() - rb0
    launches = ens.last_launches() + rebuilds * ens.rebuild_kernels()
    st = ens.state()
    qq = ens.orientations()
    # device time by phase over plain steps (each waits for the device)
    ens.set_profile(True)
    ens.step(50)
    ph, nph = ens.profile()
    ens.set_profile(False)
    ens.close()
    cpu = None
    if want_cpu:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        from bindings import EnsRestated
        o = np.argsort(st["pid"])
        x = EnsRestated(S, W, E.LAW_LINEAR, 2e-6, skin, 32, precision="f32")
        x.set_state(st["pos"][o], r, st["vel"][o], st["avel"][o])
        x.set_polyhedra(sh, so, qq[o])
        t0 = time.perf_counter()
        x.step(1)
        one = time.perf_counter() - t0
        k = max(1, min(500, int(cpu_seconds / max(one, 1e-6))))
        t0 = time.perf_counter()
        x.step(k)
        dt = time.perf_counter() - t0
        x.close()
        cpu = {"value": n * k / dt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "%d whole steps (%.1f s) of the C restatement, one thread, from the "
                         "GPU's state after its timed steps" % (k, dt)}
    rocks = so[st["pid"]] >= 0
    x, y = st["pos"][:, 0].astype(np.float64), st["pos"][:, 1].astype(np.float64)
    vt = -(x * st["vel"][:, 1] - y * st["vel"][:, 0]) / np.maximum(np.hypot(x, y), 1e-9)
    return {"workload": "ball mill mixed charge: drum and lifters as a turning mesh of %d "
                        "triangles, 30 rpm, %d steel spheres r 0.3-0.6 cm + %d convex rocks "
                        "(hulls of 8-16 points, r 0.5-1 cm), linear law + tangential history "
                        "kn 1e6 e 0.4 mu 0.6, dt 2e-6 s" % (int(S[0].ntris), n_spheres, n_rocks),
            "particles": n, "spheres": n_spheres, "polyhedra": n_rocks,
            "triangles": int(S[0].ntris), "value": n / (ms * 1e-3), "unit": UNIT,
            "ms_per_step": ms, "steps": steps, "settle_steps": settle, "skin_cm": skin,
            "cell_cm": float(S[0].cell), "block": block, "rebuilds": rebuilds,
            "gpu_launches": launches,
            "status": st["status"],
            "plain_step_ms_by_phase": {k: float(v) / max(nph, 1) for k, v in
                                       zip(("resort", "polyhedron_geometry", "polyhedron_step",
                                            "sphere_step"), ph)},
            "mean_tangential_velocity_cm_s": {"spheres": float(vt[~rocks].mean()),
                                              "rocks": float(vt[rocks].mean())},
            "cpu_baseline": cpu, "vs_cpu_port": None if not cpu else n / (ms * 1e-3) / cpu["value"]}


def case_mixed(n_spheres=100_000, n_rocks=5_000, settle=60000, steps=4):
    """The mixed charge of mill_mixed_leg: the state after `settle` graph
    steps (kept in a file under the temporary directory, so that a second run
    -- under a profiler -- starts from it at once), set again (histories
    cleared), then `steps` plain steps (one launch per kernel; steps < 8)."""
    from blaze import synth
    from blaze import ensemble as E
    S, W, p, r, sh, so, q = synth.mill_mixed_ensemble(n_spheres=n_spheres, n_rocks=n_rocks)
    path = os.path.join(tempfile.gettempdir(),
                        "blaze_mixed_%d_%d_%d.npz" % (n_spheres, n_rocks, settle))
    if not os.path.isfile(path):
        g = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=2e-6, skin=0.04, use_graph=1)
        g.set_state(p, r)
        g.set_polyhedra(sh, so, q)
        g.step(settle)
        st = g.state()
        qq = g.orientations()
        g.close()
        o = np.argsort(st["pid"])
        np.savez(path, pos=st["pos"][o], vel=st["vel"][o], avel=st["avel"][o], quat=qq[o])
    z = np.load(path)
    g = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=2e-6, skin=0.04, use_graph=1)
    g.set_state(z["pos"], r, z["vel"], z["avel"])
    g.set_polyhedra(sh, so, z["quat"])
    g.step(steps)
    status = g.sync()
    print("mixed: n %d status %d rebuilds %d" % (g.n, status, g.num_rebuilds()))
    g.close()
    return status


CASES["mixed"] = case_mixed


def c1_leg(steps=2000, warmup=20, want_cpu=True):
    """The Particles_Box plain configuration (C1): 10,000 spheres r = 0.1 cm
    falling from a jittered 20 x 20 x 25 lattice (pitch 0.3 cm) in a 10 cm
    cube of six quads, linear law kn = 1e5, e = 0.5, mu = 0.4, dt = 1e-5 s,
    gravity -981 cm/s^2 along z, the full `steps` steps from rest.  GPU: the
    reference mode (contacts-only list rebuilt every step, the reference's
    arithmetic, graph stepping) and a 0.02 cm Verlet skin, each timed with
    CUDA events over the whole run.  CPU: oracle A (the reference's kernels
    on the host) over the same full run on all host threads; its final
    state is compared with the GPU reference mode's bit for bit."""
    import torch
    from blaze import device, synth
    with tempfile.TemporaryDirectory() as d:
        P, st = synth.box_project(d)
    n = P.num_particles
    out = {"workload": "C1 Particles_Box plain: 10,000 spheres r 0.1 cm falling in a 10 cm box, "
                       "linear law kn 1e5 e 0.5 mu 0.4, dt 1e-5 s, the full run from rest",
           "particles": n, "steps": steps}
    final = {}
    for name, opts in (("reference_mode", dict(use_graph=1)),
                       ("skin", dict(skin=0.02, use_graph=1))):
        sim = device.Simulation(P, **opts)
        sim.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
        sim.prepare_graphs()
        stream = torch.cuda.ExternalStream(sim.device_state()[3])
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(steps)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b) / steps
        s_ = sim.state()
        final[name] = s_
        out[name] = {"value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                     "rebuilds": sim.num_rebuilds(), "status": device.decode_status(s_["status"])}
        sim.close()
    out["value"] = out["skin"]["value"]
    out["unit"] = UNIT
    if want_cpu:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        from bindings import RefHost, ref_available
        if ref_available():
            threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
            with _StdoutToStderr():
                R = RefHost().init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d,
                                   threads=threads, capture=False)
                R.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
                t0 = time.perf_counter()
                rc = R.step(steps)
                el = time.perf_counter() - t0
                r = R.state()
            g = final["reference_mode"]
            ig, ir = np.argsort(g["pid"]), np.argsort(r["pid"])
            same = bool(rc == 0 and all(np.array_equal(g[k][ig], r[k][ir])
                                        for k in ("pos", "vel", "avel")))
            out["cpu_baseline"] = {"value": n * steps / el, "unit": UNIT, "cores": threads,
                                   "kind": "reference",
                                   "sample": "the full %d-step run (%.1f s), reference mode"
                                             % (steps, el)}
            out["reference_mode_bit_exact_vs_cpu"] = same
            out["vs_cpu_reference"] = out["value"] / out["cpu_baseline"]["value"]
            if threads > 1:
                with _StdoutToStderr():
                    R1 = RefHost().init(P.sim_info, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d,
                                        threads=1, capture=False)
                    R1.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
                    t0 = time.perf_counter()
                    R1.step(steps)
                    e1 = time.perf_counter() - t0
                out["cpu_baseline"]["single_thread_value"] = n * steps / e1
                out["cpu_baseline"]["single_thread_sample"] = ("the full %d-step run on 1 thread "
                                                               "(%.1f s)" % (steps, e1))
    return out


def mill_leg(steps, warmup, n=100_000, skin=0.05, cpu_seconds=15.0, want_cpu=True,
             settle=60000):
    """Ball mill, the sphere charge of the mill configuration on the
    reference path: drum r = 50 cm, L = 30 cm with end plates, 30 rpm, eight
    4 x 4 cm lifters turned with the drum on the device every step
    (blaze_set_dobj_rotation), n steel spheres r ~ U[0.3, 0.6] cm in 6
    radius bins (the drum holds about 1.5e5 at lattice fill; the
    configuration's 2,000,000 such spheres would take three times the
    drum's volume), linear law kn = 1e6, e = 0.4, mu = 0.6, dt = 2e-6 s,
    rotation on, power tallies on (FP64).  The charge, packed inside the
    lifter ring, first runs `settle` untimed steps with the drum turning
    (0.12 s: it drops onto the drum and lifters and starts to tumble).
    GPU: CUDA graphs, `skin` Verlet list, `steps` timed steps after
    `warmup`; the dissipated power over the timed steps is reported.  CPU:
    the reference's kernels (oracle/_ref) with the lifter turn, all host
    threads, reference mode, a bounded sample of whole steps from the
    GPU's state and lifter positions after its timed steps."""
    import torch
    from blaze import device, synth
    with tempfile.TemporaryDirectory() as d:
        P, st = synth.mill_project(d, n=n)
    R = float(P.wobj[0].cyl_geo.radius)
    rad = float(P.mill.RadPerStep)
    sim = device.Simulation(P, skin=skin, use_graph=1)
    sim.set_cylinder_rotation(True)
    sim.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"])
    sim.set_dobj_rotation(R, R, rad)
    sim.prepare_graphs()
    sim.step(settle + max(16, -(-warmup // 8) * 8))
    status = sim.sync()
    sim.reset_energy()
    stream = torch.cuda.ExternalStream(sim.device_state()[3])
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    rb0 = sim.num_rebuilds()
    a.record(stream)
    sim.step(steps)
    b.record(stream)
    fixed = sim.last_launches()
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    rebuilds = sim.num_rebuilds() - rb0
    status |= sim.sync()
    launches = fixed + rebuilds * sim.rebuild_kernels()
    e = sim.energy()
    T = steps * float(np.float32(P.sim_info.InitalDelta_t))
    st_timed = sim.state()
    dobj_timed = sim.dobj()
    sim.close()
    out = {"workload": "ball mill: drum r 50 cm L 30 cm, 30 rpm, 8 lifters turned on the device, "
                       "%d steel spheres r 0.3-0.6 cm (6 bins), kn 1e6 e 0.4 mu 0.6, dt 2e-6 s, "
                       "rotation and power tallies on" % n,
           "particles": n, "value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
           "steps": steps, "skin_cm": skin, "rebuilds": rebuilds, "settle_steps": settle,
           "gpu_launches": launches,
           "power_w_timed_steps": {"particle": e[0] / T, "lifter": e[1] / T, "drum": e[2] / T,
                                   "total": float(e.sum()) / T},
           "status": device.decode_status(status)}
    if want_cpu:
        for k in range(P.n_d):
            P.dobj[k] = dobj_timed[k]
        cb = cpu_reference_rate(P, st_timed, cpu_seconds, hatch=False, mill=(R, R, rad))
        out["cpu_baseline"] = cb
        if cb:
            cb["sample"] += ", from the state after the GPU's timed steps"
            out["vs_cpu_reference"] = out["value"] / cb["value"]
    return out


class _StdoutToStderr:
    """Catch file descriptor 1 while the reference's kernels run (their
    printf warnings would otherwise mix with the JSON line), count the
    polyhedron kernel's penetration-clamp warnings ("large dis",
    DEM_Kernels_Compute.cuh:917-924) and pass the first lines to stderr."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.tmp = tempfile.TemporaryFile("w+b")
        os.dup2(self.tmp.fileno(), 1)
        self.large_dis = 0
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        import ctypes
        ctypes.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        self.tmp.seek(0)
        text = self.tmp.read().decode("utf-8", "replace")
        self.tmp.close()
        self.large_dis = text.count("large dis")
        if text:
            sys.stderr.write(text[:4000])
        return False


def device_status_names(st):
    from blaze import device
    return device.decode_status(st)


def silo_full_leg(steps, warmup, skin=0.04, block=256):
    """The silo discharge in the full form of the workload definition: 1,000,000
    spheres, radii uniform in [0.2, 0.4] cm, density 2600 kg/m^3, cylinder
    r = 25 cm over a 30 degree hopper of 4,096 triangles to a 6 cm outlet,
    Hertz-Mindlin (E = 1e7 Pa, nu = 0.3), restitution 0.6, mu = 0.5, rolling
    mu = 0.01, dt = 5e-6 s, FP32; one-system ensemble (tangential history,
    Coulomb cap, rolling friction, triangle walls through per-cell lists),
    CUDA graphs, Verlet skin.  Timed from the layered packing with the outlet
    open.  The reference has no Hertz-Mindlin law, history spring, rolling
    friction or triangle walls, so there is no reference arm for this line."""
    import torch
    from blaze import ensemble as E
    from blaze import synth
    S, W, p, r = synth.silo_full_ensemble(skin=skin)
    ens = E.Ensemble(S, W, law=E.LAW_HERTZ_MINDLIN, dt=5e-6, skin=skin, use_graph=1, block=block)
    ens.set_state(p, r)
    ens.step(max(3, warmup))
    status = ens.sync()
    stream = torch.cuda.ExternalStream(ens.device_state()[3])
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    rb0 = ens.num_rebuilds()
    a.record(stream)
    ens.step(steps)
    b.record(stream)
    fixed = ens.last_launches()
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    rebuilds = ens.num_rebuilds() - rb0
    launches = fixed + rebuilds * ens.rebuild_kernels()
    status |= ens.sync()
    n = ens.n
    ens.close()
    return {"workload": "silo discharge, full form: 1,000,000 spheres r U[0.2, 0.4] cm, "
                        "Hertz-Mindlin E=1e7 Pa nu=0.3 e=0.6 mu=0.5 mu_roll=0.01, "
                        "4,096-triangle hopper, dt 5e-6 s",
            "particles": n, "value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "steps": steps, "skin_cm": skin, "block": block, "rebuilds": rebuilds,
            "gpu_launches": launches, "triangles": int(S[0].ntris),
            "status": device_status_names(status),
            "cpu_baseline": None,
            "cpu_baseline_note": "the reference has no Hertz-Mindlin law, history spring, "
                                 "rolling friction or triangle walls"}


def cpu_reference_rate(P, st, seconds, max_steps=None, hatch=True, mill=None):
    """The reference's own kernels compiled as host C++ (oracle/_ref), all
    host threads, reference mode, on this workload: particle-steps/s.
    mill = (about_x, about_y, rad_per_step): drum rotating and the mill
    driver's lifter turn before every step."""
    with _StdoutToStderr() as cap:
        out = _cpu_reference_rate(P, st, seconds, max_steps, hatch, mill)
    if out is not None:
        out["large_dis_warnings"] = cap.large_dis
    return out


def _cpu_reference_rate(P, st, seconds, max_steps, hatch, mill=None):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from bindings import RefHost, ref_available
    if not ref_available():
        return None
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    si = type(P.sim_info).from_buffer_copy(bytes(P.sim_info))
    if hatch:
        si.Num_WorldObjects = P.n_w - 1  # hatch open (Device_OpenHatch drops the last object)
    R = RefHost().init(si, P.wobj, P.n_w, P.pobj, P.n_p, P.dobj, P.n_d, threads=threads,
                       capture=False)
    R.set_state(st["pos"], st["vel"], st["avel"], st["type"], st["pid"], quat=st.get("quat"))
    if mill is not None:
        R.set_cylinder_rotation(True)
        R.set_dobj_rotation(*mill)
    R.step(1)  # first step outside the clock (page-in)
    steps = 0
    t0 = time.perf_counter()
    while True:
        R.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or (max_steps and steps >= max_steps):
            break
    out = {"value": P.num_particles * steps / el, "unit": UNIT, "cores": threads,
           "kind": "reference",
           "sample": "%d full steps of the %d-particle workload (%.1f s), reference mode"
                     % (steps, P.num_particles, el)}
    if threads > 1:
        # the same kernels on one host thread, a third of the time budget (20 s at most)
        R.lib.refh_set_threads(1)
        s1 = 0
        t0 = time.perf_counter()
        while True:
            R.step(1)
            s1 += 1
            e1 = time.perf_counter() - t0
            if e1 >= min(seconds / 3.0, 20.0) or (max_steps and s1 >= max_steps):
                break
        out["single_thread_value"] = P.num_particles * s1 / e1
        out["single_thread_sample"] = "%d further full steps on 1 thread (%.1f s)" % (s1, e1)
    return out


def run_reference_arm(args, rank):
    if rank != 0:
        return 0
    with tempfile.TemporaryDirectory() as d:
        P, st = make_workload(d, args.n)
        budget = max(10.0, min(150.0, 0.5 * (args.steps + args.warmup)))
        cb = cpu_reference_rate(P, st, budget, max_steps=args.steps)
    if cb is not None:
        # The GPU arm times the bed after 48,000 untimed settling steps; the
        # host cores would need hours for them, so the reference's kernels
        # are timed on the generated packing of the same workload.  On a
        # 20,000-sphere silo they ran 15 % faster there than on the settled
        # bed (10.8 vs 9.3 M particle-steps/s), so this arm is, if anything,
        # favoured.
        cb["sample"] += (", from the generated packing (the settling pre-roll is not run on the "
                         "host cores)")
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libblaze_refhost.so not built (reference tree absent at build)"}))
        return 0
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config(args), "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)

    import torch
    import torch.distributed as dist
    from blaze import device

    torch.cuda.set_device(local)
    if args.case:
        rc = CASES[args.case[0]](*[int(a) for a in args.case[1:]])
        return 1 if rc else 0
    if args.silo_full_only:
        print(json.dumps(silo_full_leg(args.silo_full_steps, args.warmup)))
        return 0
    if args.mill_only:
        print(json.dumps(mill_leg(args.mill_steps, args.warmup, cpu_seconds=args.cpu_seconds,
                                  want_cpu=not args.no_cpu_baseline)))
        return 0
    if args.mill_mixed_only:
        print(json.dumps(mill_mixed_leg(args.mill_steps, args.warmup, cpu_seconds=args.cpu_seconds,
                                        want_cpu=not args.no_cpu_baseline)))
        return 0
    if args.poly_only:
        print(json.dumps(poly_leg(args.poly_steps, args.warmup, cpu_seconds=args.cpu_seconds,
                                  want_cpu=not args.no_cpu_baseline)))
        return 0
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    tmp = tempfile.TemporaryDirectory()
    P, st0 = make_workload(tmp.name, args.n)
    n = P.num_particles

    # The generated packing (size-banded simple-cubic layers) rains onto the
    # hopper for its first ~10,000 steps: contacts per particle fall from ~5
    # to ~0 and rise again.  The timed discharge starts from the settled bed
    # (untimed, deterministic: the same state every run), where the cost per
    # step is steady.
    sim = device.Simulation(P, skin=args.skin, max_nbr=args.max_nbr, use_graph=1)
    sim.set_state(st0["pos"], st0["vel"], st0["avel"], st0["type"], st0["pid"])
    sim.prepare_graphs()
    t_settle = time.perf_counter()
    sim.step(args.settle_steps)
    status = sim.sync()
    t_settle = time.perf_counter() - t_settle
    settled = sim.state()
    st = dict(pos=settled["pos"], vel=settled["vel"], avel=settled["avel"],
              type=settled["type"], pid=settled["pid"])
    sim.open_hatch()  # the discharge: the last world object (hatch) is dropped
    fast = 1 if args.law == "fast" else 0
    sim.set_options(skin=args.skin, max_nbr=args.max_nbr, use_graph=1, fast_law=fast)
    # every graph is instantiated before the timed region; the warm-up runs
    # at least W steps and ends on a block start (a multiple of 8 steps past
    # the 8 checked steps that follow a change of options), so the timed
    # region opens with a whole block
    sim.prepare_graphs()
    warm = max(16, -(-args.warmup // 8) * 8)
    sim.step(warm)
    status |= sim.sync()
    stream = torch.cuda.ExternalStream(sim.device_state()[3])
    contacts0 = contacts_per_particle(sim)

    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    phys = vis.split(",")[local] if vis else str(local)
    sampler = ClockSampler(phys)
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    rb0 = sim.num_rebuilds()
    x0 = sim.num_exact_blocks()
    e0.record(stream)
    sim.step(args.steps)
    e1.record(stream)
    fixed_launches = sim.last_launches()
    e1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    rebuilds = sim.num_rebuilds() - rb0
    exact_blocks = sim.num_exact_blocks() - x0
    # unconditional launches + re-sort bodies + the exact mode's extra gate
    launches = fixed_launches + rebuilds * sim.rebuild_kernels() + exact_blocks
    status |= sim.sync()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = n * world * args.steps / (ms * 1e-3)

    # per-kernel timing for the roofline (separate pass, same workload; the
    # event-timed path steps without the graph), for both forms of the law
    kstep = {}
    for law in ("exact", "fast"):
        sim.set_options(skin=args.skin, max_nbr=args.max_nbr, use_graph=1,
                        fast_law=1 if law == "fast" else 0)
        sim.step(16)
        sim.set_profile(True)
        sim.step(min(max(args.steps, 16), 200))
        ms_rebuild, ms_step, nsteps = sim.profile()
        sim.set_profile(False)
        kstep[law] = ms_step / max(nsteps, 1)
    t_step = kstep[args.law] * 1e-3
    peak, peak_kind = peak_hbm()
    achieved = n * B_ALG / t_step / 1e9
    traffic, traffic_n = ncu_traffic()
    if traffic is not None and traffic_n:
        traffic = traffic * n / traffic_n

    # reference mode (rebuild every step, the reference's arithmetic) for context
    sim.set_options(skin=0.0, use_graph=1, fast_law=0)
    sim.step(3)
    sim.sync()
    r0 = torch.cuda.Event(enable_timing=True)
    r1 = torch.cuda.Event(enable_timing=True)
    kref = min(args.steps, 400)
    r0.record(stream)
    sim.step(kref)
    r1.record(stream)
    r1.synchronize()
    ref_mode_value = n * kref / (r0.elapsed_time(r1) * 1e-3)
    sim.close()

    # end to end through the reference-facing C ABI with host buffers
    lib = device.load()
    kd = device.KDevice(P.wobj, P.pobj, P.dobj, P.n_w, P.n_p, P.n_d, P.sim_info, P.init)
    kd.IDevice_OpenHatch(P.wobj, P.n_w)
    hp = torch.empty((n, 3), dtype=torch.float32).pin_memory().numpy()
    hv = torch.empty((n, 3), dtype=torch.float32).pin_memory().numpy()
    hw = torch.empty((n, 3), dtype=torch.float32).pin_memory().numpy()
    ht = torch.empty(n, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    hi = torch.empty(n, dtype=torch.int32).pin_memory().numpy()
    hp[:] = st["pos"]; hv[:] = st["vel"]; hw[:] = st["avel"]; ht[:] = st["type"]; hi[:] = st["pid"]
    kd.IDevice_Set_ParticleSystem_State(hp, None, hv, hw, None, ht, hi)
    kd.IDevice_DEM_UpdateSim()
    kd.IDevice_Get_System_State(hp, None, hv, hw, None, ht, hi)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        kd.IDevice_Set_ParticleSystem_State(hp, None, hv, hw, None, ht, hi)
        kd.IDevice_DEM_UpdateSim()
        kd.IDevice_Get_System_State(hp, None, hv, hw, None, ht, hi)
    el = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([el], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el = float(t.item())
    kd.clean()
    e2e_value = n * world * args.e2e_steps / el
    state_bytes = n * (12 + 12 + 12 + 4 + 4)

    silo_full = None
    if not args.no_silo_full:
        silo_full = silo_full_leg(args.silo_full_steps, args.warmup)
    poly = None
    if not args.no_poly:
        poly = poly_leg(args.poly_steps, args.warmup, cpu_seconds=args.cpu_seconds,
                        want_cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)
    mill = None
    if not args.no_mill:
        mill = mill_leg(args.mill_steps, args.warmup, cpu_seconds=args.cpu_seconds,
                        want_cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)
    mill_mesh = None
    if not args.no_mill_mesh:
        mill_mesh = mill_mesh_leg(args.mill_steps, args.warmup)
    mill_mixed = None
    if not args.no_mill_mixed:
        mill_mixed = mill_mixed_leg(args.mill_steps, args.warmup, cpu_seconds=args.cpu_seconds,
                                    want_cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)
    c1 = None
    if not args.no_c1:
        c1 = c1_leg(2000, args.warmup, want_cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)
    batched = None
    if not args.no_batched:
        batched = batched_leg(args.batched_steps, args.warmup)
    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_leg(args.adjoint_steps)

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_reference_rate(P, st, args.cpu_seconds)
        if cb:
            cb["sample"] += ", from the settled bed the GPU arm times"

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(args),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "steps": args.e2e_steps,
                    "path": "Device_Set_System_State + Device_DEM_UpdateSim + "
                            "Device_Get_System_State per step, pinned host buffers"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "k_step (fused contact + walls + integration)",
                         "peak_source": peak_kind,
                         "bytes_per_launch": n * B_ALG, "launch_ms": t_step * 1e3},
            "cpu_baseline": cb,
            "gpu_launches": launches,
            "clocks": clocks,
            "law": args.law,
            "timed_from": "the settled bed (%d untimed steps with the hatch closed, %.1f s), "
                          "hatch open, %d warm-up steps" % (args.settle_steps, t_settle, warm),
            "contacts_per_particle": contacts0,
            "k_step_ms": kstep,
            "rebuilds_in_timed_region": rebuilds,
            "exact_blocks_in_timed_region": exact_blocks,
            "rebuild_ms_per_step": ms_rebuild / max(nsteps, 1),
            "reference_mode_value": ref_mode_value,
            "silo_full": silo_full,
            "polyhedra": poly,
            "mill": mill,
            "mill_mesh": mill_mesh,
            "mill_mixed": mill_mixed,
            "c1_box": c1,
            "batched": batched,
            "adjoint": adjoint,
            "status": device.decode_status(status),
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    tmp.cleanup()
    return 0


if __name__ == "__main__":
    sys.exit(main())
