"""GPU mixed charge (spheres and convex polyhedra in one system,
blaze_ens_set_polyhedra) against the C restatement (oracle/ens_oracle.c).

Cases (seeded, synth):
  box   300 steel balls r ~ U[0.3, 0.6] cm and 24 rocks (hulls of 8-16
        points on spheres of radius 0.5-1 cm) in a closed box of planes,
        linear law kn 1e5, e 0.4, mu 0.6, dt 1e-5 s: poured from rest onto
        the floor and each other
  drum  400 balls and 24 rocks in a small turning drum of triangles (r 12 cm,
        L 8 cm, 48 x 6 barrel quads, 4 lifters, end plates as turning planes),
        30 rpm
The bar: the GPU state (positions, velocities, spins, orientations) equals
the FP32 restatement's bit for bit at every checkpoint; the contact forces
of one step from a common state equal the FP64 restatement's within 1e-5 of
each particle's force scale (the larger of its contact force and weight).
"""
import numpy as np
import pytest

from bindings import EnsRestated
from blaze import ensemble as E
from blaze import synth

pytestmark = pytest.mark.gpu

DT = 1e-5
SKIN = 0.04


def box_case():
    return synth.mixed_box_ensemble(n_spheres=300, n_rocks=24, kn=1e5)


def drum_case():
    return synth.mill_mixed_ensemble(n_spheres=400, n_rocks=24, R=12.0, L=8.0, n_seg=48,
                                     n_len=6, n_lifters=4, lifter_w=2.0, lifter_h=2.0, kn=1e5)


CASES = {"box": box_case, "drum": drum_case}


def by_pid(st, q):
    o = np.argsort(st["pid"])
    return (st["pos"][o], st["vel"][o], st["avel"][o], q[o])


def run_both(case, checkpoints, use_graph=1):
    S, W, p, r, sh, so, q = case
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=DT, skin=SKIN, use_graph=use_graph)
    ens.set_state(p, r)
    ens.set_polyhedra(sh, so, q)
    o = EnsRestated(S, W, E.LAW_LINEAR, DT, SKIN, 32, precision="f32")
    o.set_state(p, r)
    o.set_polyhedra(sh, so, q)
    done = 0
    out = []
    for c in checkpoints:
        ens.step(c - done)
        o.step(c - done)
        done = c
        g = ens.state()
        assert g["status"] == 0, g["status"]
        h = o.state()
        assert h["status"] == 0, h["status"]
        out.append((c, by_pid(g, ens.orientations()), by_pid(h, o.orientations()),
                    ens.num_rebuilds(), o.num_rebuilds()))
    ens.close()
    o.close()
    return out


CHECKPOINTS = {"box": [1, 50, 2000, 8000, 20000], "drum": [1, 50, 2000, 8000, 20000]}


@pytest.mark.parametrize("name", ["box", "drum"])
def test_mixed_charge_bit_exact(name):
    case = CASES[name]()
    res = run_both(case, CHECKPOINTS[name])
    so = case[5]
    for c, g, h, rg, rh in res:
        names = ("position", "velocity", "spin", "orientation")
        bad = [nm for nm, a, b in zip(names, g, h) if not np.array_equal(a.astype(np.float64), b)]
        moved = float(np.abs(g[0] - case[2]).max())
        print("%s step %d: re-sorts GPU %d restatement %d, largest displacement %.3f cm, %s"
              % (name, c, rg, rh, moved, "bit-exact" if not bad else "differs: " + ", ".join(bad)))
        assert rg == rh
        assert not bad, (c, bad)


def test_mixed_box_graph_and_plain_agree():
    case = box_case()
    S, W, p, r, sh, so, q = case
    outs = []
    for ug in (0, 1):
        ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=DT, skin=SKIN, use_graph=ug)
        ens.set_state(p, r)
        ens.set_polyhedra(sh, so, q)
        ens.step(3000)
        outs.append(by_pid(ens.state(), ens.orientations()))
        ens.close()
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", ["box", "drum"])
def test_mixed_forces_against_fp64(name):
    """From the GPU's state after 12,000 steps (a bed in contact), one step
    on the GPU with forces captured and one of the FP64 restatement from the
    same state (histories start empty on both)."""
    S, W, p, r, sh, so, q = CASES[name]()
    ens = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=DT, skin=SKIN, use_graph=1)
    ens.set_state(p, r)
    ens.set_polyhedra(sh, so, q)
    ens.step(12000)
    st = ens.state()
    qq = ens.orientations()
    ens.close()
    o = np.argsort(st["pid"])
    pos, vel, avel, quat = st["pos"][o], st["vel"][o], st["avel"][o], qq[o]
    g = E.Ensemble(S, W, law=E.LAW_LINEAR, dt=DT, skin=SKIN, use_graph=0, capture_forces=1)
    g.set_state(pos, r, vel, avel)
    g.set_polyhedra(sh, so, quat)
    g.step(1)
    fg, tg = g.forces()
    sg = g.state()
    g.close()
    og = np.argsort(sg["pid"])
    fg, tg = fg[og].astype(np.float64), tg[og].astype(np.float64)
    x = EnsRestated(S, W, E.LAW_LINEAR, DT, SKIN, 32, precision="f64")
    x.set_state(pos, r, vel, avel)
    x.set_polyhedra(sh, so, quat)
    x.step(1)
    fx, tx = x.forces()
    sx = x.state()
    x.close()
    ox = np.argsort(sx["pid"])
    fx, tx = fx[ox], tx[ox]
    rho_s = S[0].density
    mass = np.where(so < 0, rho_s * 4.0 / 3.0 * np.pi * r.astype(np.float64) ** 3, 0.0)
    for k in np.nonzero(so >= 0)[0]:
        mass[k] = E.mass_properties(sh[so[k]])[0]
    gmag = np.linalg.norm(np.array([S[0].gravity[i] for i in range(3)]))
    scale = np.maximum(np.linalg.norm(fx, axis=1), mass * gmag)
    ef = np.linalg.norm(fg - fx, axis=1) / scale
    # torques: scale by force scale x bounding radius
    et = np.linalg.norm(tg - tx, axis=1) / (scale * r)
    rocks = so >= 0
    touching = np.linalg.norm(fx, axis=1) > 0
    print("%s: %d of %d particles in contact (%d rocks); force error vs FP64: spheres %.2e, "
          "rocks %.2e; torque %.2e" % (name, touching.sum(), len(so), (touching & rocks).sum(),
                                      ef[~rocks].max(), ef[rocks].max(), et.max()))
    assert (touching & rocks).sum() >= 5   # rock contacts covered (7-17 in these cases)
    assert ef.max() < 1e-5 and et.max() < 1e-5


def test_set_polyhedra_rejections():
    """blaze_ens_set_polyhedra refuses what the mixed step does not cover,
    with -1 and the ensemble left usable: after a step; a law other than
    the linear one; a bounding radius that does not fit the cells; an
    invalid hull."""
    from blaze import device
    S, W, p, r, sh, so, q = box_case()

    def fresh(**kw):
        ens = E.Ensemble(S, W, dt=DT, skin=SKIN, use_graph=0, **kw)
        ens.set_state(p, r)
        return ens

    ens = fresh()
    ens.step(1)
    with pytest.raises(device.BlazeError):
        ens.set_polyhedra(sh, so, q)          # not right after set_state
    ens.set_state(p, r)
    ens.set_polyhedra(sh, so, q)              # fine again after set_state
    ens.step(2)
    assert ens.sync() == 0
    ens.close()
    ens = fresh(law=E.LAW_HERTZ_MINDLIN)
    with pytest.raises(device.BlazeError):
        ens.set_polyhedra(sh, so, q)
    ens.close()
    big = list(sh)
    v = np.asarray(sh[0].verts).reshape(-1, 3)[:sh[0].nverts] * 3.0   # 3x the size: too big for a cell
    f = np.asarray(sh[0].faces).reshape(-1, 3)[:sh[0].nfaces]
    big[0] = E.shape(v, f, sh[0].density)
    ens = fresh()
    with pytest.raises(device.BlazeError):
        ens.set_polyhedra(big, so, q)
    bad = list(sh)
    bad[0] = E.shape(v / 3.0, f[:, [0, 2, 1]], sh[0].density)            # inside out
    with pytest.raises(device.BlazeError):
        ens.set_polyhedra(bad, so, q)
    ens.set_polyhedra(sh, so, q)
    ens.step(2)
    assert ens.sync() == 0
    ens.close()
