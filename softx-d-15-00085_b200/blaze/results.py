"""The reference driver's result files (main.cpp), written through the
library: FlowRate.dat of a silo run and Results.dat of a ball-mill run.

silo_discharge() is main.cpp's headless silo loop (main.cpp:1068-1078 with
UpdateSim's flow counter, main.cpp:133-147): the counter starts at zero and
every `flow_steps` steps, before the next step, Silo_Stats counts the
particles above the hatch (blaze_count_above, on the device) and a line
"time percent-discharged" is appended; the time is the double sum of the
float step, as the driver accumulates it (main.cpp:236)."""
import ctypes as C

import numpy as np

from . import device


def write_flow_line(path, time, n0, remaining):
    """Append main.cpp:142's line: time and percent of `n0` below the hatch."""
    device._check(device.load().blaze_write_flow_line(path.encode(), float(time), int(n0),
                                                      int(remaining)), "blaze_write_flow_line")


def write_power_line(path, time, energy3, steps_per_rev, dt):
    """Append main.cpp:74-82's line: the revolution's particle, lifter and
    drum energies (Device_Get_Energy's first three) over its duration."""
    e = np.ascontiguousarray(energy3, np.float32)
    device._check(device.load().blaze_write_power_line(
        path.encode(), float(time), e.ctypes.data_as(C.POINTER(C.c_float)), int(steps_per_rev),
        float(dt)), "blaze_write_power_line")


def silo_discharge(sim, project, steps, path=None, t0=0.0):
    """Step a silo run whose hatch is open for `steps` steps and record the
    discharge as the reference's driver does: every project.silo.flow_steps
    steps the percentage of the initial particles that left (below the
    hatch).  `t0` is the driver's clock when the hatch opened.  Returns
    [(time, percent)]; with `path`, appends the lines of FlowRate.dat there."""
    fs = int(project.silo.flow_steps)
    h = float(project.silo.hatch_height)
    n0 = int(project.num_particles)
    dt = float(np.float32(project.sim_info.InitalDelta_t))
    t, k, out = float(t0), 0, []
    while k + fs <= steps:
        sim.step(fs)
        k += fs
        for _ in range(fs):
            t += dt
        rem = sim.count_above(h)
        if path is not None:
            write_flow_line(path, t, n0, rem)
        out.append((t, float(np.float32(n0 - rem) / np.float32(n0)) * 100.0))
    return out
