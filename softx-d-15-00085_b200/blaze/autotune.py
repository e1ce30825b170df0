"""Autotuner of the ensemble path: picks the Verlet skin (and with it the
cell size, 2 r_max + skin) and the thread-block size of the step kernel by
timing short runs of the caller's own workload on the GPU.

A larger skin re-sorts less often but tests more neighbour candidates each
step; the best trade depends on how fast the particles move and on how many
systems share the re-sort (any particle of any system triggers it), so it is
measured, not modelled.  Each trial steps a fresh ensemble from the given
state and is timed with CUDA events on the ensemble's stream.
"""
import math

import numpy as np

from . import ensemble as E

SKINS = (0.01, 0.02, 0.04, 0.08)
BLOCKS = (128, 256, 512)


def regrid(systems, skin, r_max):
    """Copies of `systems` with cell = 2 r_max + skin and the grid grown or
    shrunk to cover the same box (origin kept)."""
    out = []
    cell = 2.0 * r_max + skin
    for s in systems:
        c = E.System.from_buffer_copy(bytes(s))
        for k in range(3):
            extent = s.ncells[k] * s.cell
            c.ncells[k] = max(1, int(math.ceil(extent / cell)))
        c.cell = cell
        out.append(c)
    return out


def _time(systems, walls, pos, radius, vel, opts, steps, warmup):
    import torch
    e = E.Ensemble(systems, walls, **opts)
    try:
        e.set_state(pos, radius, vel)
        e.step(warmup)
        e.sync()
        stream = torch.cuda.ExternalStream(e.device_state()[3])
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e.step(steps)
        b.record(stream)
        b.synchronize()
        status = e.sync()
        return a.elapsed_time(b) / steps, status
    finally:
        e.close()


def preroll(systems, walls, pos, radius, vel, steps, *, law, dt, max_nbr, skin=0.02):
    """State after `steps` steps with a default skin, in the caller's order
    (trials then start where the particles already move as they will)."""
    r_max = float(np.max(radius))
    e = E.Ensemble(regrid(systems, skin, r_max), walls, law=law, dt=dt, skin=skin,
                   max_nbr=max_nbr, use_graph=1)
    try:
        e.set_state(pos, radius, vel)
        e.step(steps)
        st = e.state()
    finally:
        e.close()
    order = np.argsort(st["pid"])
    return st["pos"][order], st["vel"][order]


def tune(systems, walls, pos, radius, vel=None, *, law=E.LAW_LINEAR, dt=1e-5, max_nbr=32,
         skins=SKINS, blocks=BLOCKS, steps=200, warmup=8, preroll_steps=600):
    """Returns (best, trials): best = dict(skin, cell, block, ms_per_step,
    systems) with the re-gridded systems to create the ensemble with, and
    trials the list of (skin, block, ms_per_step, status) measured.  The
    trials start from the state after `preroll_steps` steps, so re-sorts
    happen at the rate the run will see.  Trials whose run raised a status
    bit (list overflow, particle outside the grid) are not chosen."""
    r_max = float(np.max(radius))
    if preroll_steps > 0:
        pos, vel = preroll(systems, walls, pos, radius, vel, preroll_steps, law=law, dt=dt,
                           max_nbr=max_nbr)
    trials = []
    best = None
    for skin in skins:
        S = regrid(systems, skin, r_max)
        opts = dict(law=law, dt=dt, skin=skin, max_nbr=max_nbr, use_graph=1, block=256)
        ms, st = _time(S, walls, pos, radius, vel, opts, steps, warmup)
        trials.append((skin, 256, ms, st))
        if st == 0 and (best is None or ms < best["ms_per_step"]):
            best = dict(skin=skin, cell=2.0 * r_max + skin, block=256, ms_per_step=ms, systems=S)
    if best is None:
        raise RuntimeError("autotune: every trial raised a status bit: %r" % trials)
    for blk in blocks:
        if blk == 256:
            continue
        opts = dict(law=law, dt=dt, skin=best["skin"], max_nbr=max_nbr, use_graph=1, block=blk)
        ms, st = _time(best["systems"], walls, pos, radius, vel, opts, steps, warmup)
        trials.append((best["skin"], blk, ms, st))
        if st == 0 and ms < best["ms_per_step"]:
            best = dict(best, block=blk, ms_per_step=ms)
    return best, trials
