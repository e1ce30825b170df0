"""Statistics of long runs, computed the same way from oracle A's states
(tests/golden/make_long_run.py) and from the library's (the long-run GPU
tests)."""
import numpy as np

# central columns of the 10 cm box, clear of the side walls, and the slabs
BOX_XY = (1.0, 9.0)
SLAB = 0.5
SLABS = np.arange(0.0, 10.0 + 1e-9, SLAB)


def kinetic_energy(vel, avel, mass, radius):
    """Translational + rotational kinetic energy of equal spheres
    (moment of inertia 0.4 m r^2), in the project's units."""
    v = np.asarray(vel, np.float64)
    w = np.asarray(avel, np.float64)
    return 0.5 * mass * float((v * v).sum()) + 0.2 * mass * radius * radius * float((w * w).sum())


def solid_fraction_profile(pos, radius, xy=BOX_XY, edges=SLABS, axis=2):
    """Solid fraction in horizontal slabs of the central columns: the volume
    of each sphere (centre inside the columns) between the slab's planes,
    summed and divided by the slab's volume."""
    p = np.asarray(pos, np.float64)
    h = [a for a in range(3) if a != axis]
    inside = np.all((p[:, h] >= xy[0]) & (p[:, h] <= xy[1]), axis=1)
    z = p[inside, axis]
    r = float(radius)

    def cap(t):  # volume of the sphere below height zc + t
        t = np.clip(t, -r, r)
        return np.pi * (r * r * t - t ** 3 / 3.0) + 2.0 / 3.0 * np.pi * r ** 3

    out = []
    for a, b in zip(edges[:-1], edges[1:]):
        vol = cap(b - z) - cap(a - z)
        out.append(vol.sum() / ((xy[1] - xy[0]) ** 2 * (b - a)))
    return np.array(out)


def discharged_percent(above, n0):
    """main.cpp:142: the percentage of the initial particles below the hatch,
    in float as the driver forms it."""
    a = np.asarray(above)
    return (np.float32(n0) - a.astype(np.float32)) / np.float32(n0) * 100.0
