"""Calibration harness: the ensemble forward run and its reverse sweep
(include/blaze_ens.h, reverse mode) as a torch.autograd.Function, so a loss
written in torch on the final state gets gradients with respect to the
contact-law parameters (kn, restitution, mu, mu_wall per system) and the
initial velocities.

The workload is the calibration configuration: independent systems of
spheres settling into square-base boxes; the loss compares each system's
settled bed height and the normal-force profile on one side wall (32 height
bins) with targets from a run with hidden parameters.
"""
import math

import numpy as np
import torch

from . import ensemble as E
from . import synth

PARAMS = ("kn", "restitution", "mu", "mu_wall")


def calibration_ensemble(nsys=64, n=20000, base=5.0, r_min=0.1, r_max=0.2, rho=2500.0,
                         kn=1e5, restitution=0.5, mu=0.4, skin=0.02, seed=4):
    """nsys systems of n spheres (radii uniform in [r_min, r_max] cm, seed)
    in boxes of square base `base` cm, tall enough for the loose initial FCC
    lattice; linear law with tangential history (kt = 2/7 kn).  Returns
    (systems, walls, pos, radius)."""
    rng = np.random.default_rng(seed)
    density = rho * 1e-6
    cell = 2.0 * r_max + skin
    pitch = 2.0 * r_max + 0.5 * skin
    # height for n sites of the FCC lattice (4 sites per a^3), with margin
    a = pitch * math.sqrt(2.0)
    per_layer = 2.0 * ((base - 2 * r_max) / a + 1) ** 2
    H = (n / per_layer + 2) * a / 2.0 * 1.15 + 2 * r_max + 1.0
    systems, walls, pos, rad = [], [], [], []
    jitter = 0.2 * (pitch - 2 * r_max)
    probe = np.random.default_rng(0)
    while True:  # grow the box until the lattice holds n spheres
        try:
            synth.lattice_fill(n, (r_max + 0.01,) * 3,
                               (base - r_max - 0.01, base - r_max - 0.01, H - r_max - 0.01),
                               pitch, probe)
            break
        except ValueError:
            H *= 1.1
    for s in range(nsys):
        r = rng.uniform(r_min, r_max, size=n)
        p = synth.lattice_fill(n, (r_max + 0.01, r_max + 0.01, r_max + 0.01),
                               (base - r_max - 0.01, base - r_max - 0.01, H - r_max - 0.01),
                               pitch, rng, jitter=jitter)
        systems.append(synth.box_system(n, base, H, cell, len(walls), density=density, kn=kn,
                                        restitution=restitution, mu=mu))
        walls += synth.box_walls(base, H)
        pos.append(p.astype(np.float32))
        rad.append(r.astype(np.float32))
    return systems, walls, np.concatenate(pos), np.concatenate(rad)


def initial_velocity(n, seed=4, spread=30.0, down=50.0):
    """Initial velocities of a calibration run (cm/s): normal with standard
    deviation `spread` per component plus `down` towards the floor, so
    neighbours and walls are hit from the first steps."""
    rng = np.random.default_rng(seed + 1000)
    v = rng.normal(scale=spread, size=(n, 3))
    v[:, 2] -= down
    return v


def with_params(systems, params):
    """Copies of `systems` with (kn, restitution, mu, mu_wall) from the rows
    of `params` (nsys x 4)."""
    out = []
    for s, row in zip(systems, np.asarray(params, np.float64)):
        c = E.System.from_buffer_copy(bytes(s))
        c.kn, c.restitution, c.mu, c.mu_wall = (float(x) for x in row)
        out.append(c)
    return out


class Runner:
    """One ensemble, its reverse mode and the initial state of a
    calibration run of `nsteps` steps with checkpoints every `segment`.

    window: reverse only the last `window` steps (truncated
    backpropagation, Adjoint.backward).  The pathwise derivative of a
    settling run grows about 5 % per step (dense granular flow is chaotic),
    so over a 3,000-step run the full reverse sweep overflows FP32 and
    carries no usable slope; a window of ~50 steps gives the derivative of
    the final steps' response to the law constants, bounded and checked
    against finite differences (tests/test_adjoint_oracle.py).  With a
    window the gradient with respect to the initial velocities is zero (the
    state before the window is held fixed)."""

    def __init__(self, systems, walls, pos, radius, nsteps, segment=100, dt=1e-5, skin=0.02,
                 max_nbr=32, tape_bytes=0, window=None):
        self.systems = systems
        self.walls = walls
        self.pos0 = np.ascontiguousarray(pos, np.float32)
        self.radius = np.ascontiguousarray(radius, np.float32)
        self.ens = E.Ensemble(systems, walls, law=E.LAW_LINEAR, dt=dt, skin=skin,
                              max_nbr=max_nbr, use_graph=0)
        self.adj = E.Adjoint(self.ens, nsteps, segment, tape_bytes)
        self.cur = systems
        self.window = window

    def close(self):
        self.adj.close()
        self.ens.close()


class EnsembleRun(torch.autograd.Function):
    """(params nsys x 4, v0 N x 3) -> (final positions N x 3, final
    velocities N x 3), rows in the order of the initial state; float64
    tensors on the CPU."""

    @staticmethod
    def forward(ctx, params, v0, runner):
        runner.cur = with_params(runner.systems, params.detach().cpu().numpy())
        runner.ens.set_params(runner.cur)
        runner.ens.set_state(runner.pos0, runner.radius, v0.detach().cpu().numpy())
        status = runner.adj.forward()
        if status:
            raise RuntimeError("forward raised status bits %d" % status)
        st = runner.ens.state()
        order = np.argsort(st["pid"])
        ctx.runner = runner
        ctx.pid = st["pid"]
        return (torch.from_numpy(st["pos"][order].astype(np.float64)),
                torch.from_numpy(st["vel"][order].astype(np.float64)))

    @staticmethod
    def backward(ctx, gpos, gvel):
        r = ctx.runner
        pid = ctx.pid
        gx = gpos.detach().cpu().numpy()[pid]
        gv = gvel.detach().cpu().numpy()[pid]
        _, gv0, _, gc = r.adj.backward(gx, gv, None, window=r.window)
        gu = E.user_param_grads(gc, r.cur)          # kn, kt_ratio, e, mu, mu_wall
        gparams = torch.from_numpy(gu[:, [0, 2, 3, 4]].copy())
        if r.window is not None and r.window < r.adj.nsteps:
            gv0 = np.zeros_like(gv0)                # the state before the window is fixed
        return gparams, torch.from_numpy(gv0.astype(np.float64)), None


def system_slices(systems):
    off = np.concatenate([[0], np.cumsum([s.n for s in systems])])
    return [slice(int(off[k]), int(off[k + 1])) for k in range(len(systems))]


def observables(pos, vel, params, systems, radius, base=5.0, nbins=32):
    """Per system: bed height (mean sphere height) and the normal-force
    profile on the wall x = 0 in `nbins` height bins (linear law: kn d -
    c_n v_n with c_n = 2 beta(e) sqrt(m kn), d the overlap)."""
    rad = torch.as_tensor(radius, dtype=torch.float64)
    heights, profiles = [], []
    for s, sl in enumerate(system_slices(systems)):
        S = systems[s]
        kn, e = params[s, 0], params[s, 1]
        le = torch.log(e)
        beta2 = 2.0 * (-le / torch.sqrt(le * le + math.pi ** 2))
        x = pos[sl, 0]
        z = pos[sl, 2]
        r = rad[sl]
        heights.append(z.mean())
        m = S.density * 4.0 / 3.0 * math.pi * r ** 3
        delta = r - x
        fn = kn * delta - beta2 * torch.sqrt(m * kn) * vel[sl, 0]
        touch = (delta > 0).to(torch.float64)
        H = S.ncells[2] * S.cell
        b = torch.clamp((z.detach() / H * nbins).long(), 0, nbins - 1)
        prof = torch.zeros(nbins, dtype=torch.float64).index_add(0, b, fn * touch)
        profiles.append(prof)
    return torch.stack(heights), torch.stack(profiles)


def loss_fn(pos, vel, params, systems, radius, target):
    """Mean squared error of bed height (cm) and of the wall-force profile
    (scaled by the target's largest force) against target = (h*, P*)."""
    h, P = observables(pos, vel, params, systems, radius)
    h_t, P_t = target
    scale = torch.clamp(P_t.abs().max(), min=1e-12)
    return ((h - h_t) ** 2).mean() + (((P - P_t) / scale) ** 2).mean()
