"""The driver's result lines (FlowRate.dat, Results.dat) as the library
writes them, against the reference's expressions (main.cpp:142, 74-82:
float arithmetic, ostream's default six significant digits) restated in
numpy.  No GPU needed."""
import os

import numpy as np

from blaze import results


def ref_flow(time, n0, rem):
    pct = float(np.float32(n0 - rem) / np.float32(n0)) * 100.0
    return "%g %g\n" % (time, pct)


def ref_power(time, e, steps, dt):
    e = np.asarray(e, np.float32)
    T = np.float32(steps) * np.float32(dt)
    tot = np.float32(np.float32(e[0] + e[1]) + e[2]) / T
    return "time: %g Power:   Total = %g  Particle: %g  Lifter: %g Drum %g\n" % (
        time, tot, e[0] / T, e[1] / T, e[2] / T)


def test_flow_lines(tmp_path):
    path = str(tmp_path / "FlowRate.dat")
    cases = [(0.01, 1950, 1950), (0.0200000009, 1950, 1949), (1.23456789, 1000000, 333333),
             (7.5, 7, 0), (1e-5 * 37, 12345, 12000)]
    for c in cases:
        results.write_flow_line(path, *c)
    lines = open(path).readlines()
    assert lines == [ref_flow(*c) for c in cases], lines


def test_power_lines(tmp_path):
    path = str(tmp_path / "Results.dat")
    rng = np.random.default_rng(2)
    cases = []
    for k in range(20):
        e = rng.uniform(1e-3, 1e3, 3).astype(np.float32)
        cases.append((float(k + 1) * 2.72727, e, int(rng.integers(1000, 300000)), 1e-5))
    for c in cases:
        results.write_power_line(path, *c)
    lines = open(path).readlines()
    assert lines == [ref_power(*c) for c in cases]
    assert os.path.getsize(path) > 0
